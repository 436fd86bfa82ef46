"""K1 (pattern) and K2 (scatter map) on the GPU against the reference's own outputs (golden
fixtures) and against the oracle at larger sizes: bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_pattern_and_map_match_reference(fb, name):
    z, meta = golden(name)
    N, k = int(meta["N"]), int(meta["k"])
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="dirichlet")
    assert np.array_equal(V.cell_dofs.ravel(), z["cell_dofs"])
    P = V.pattern()
    ip, ix = P.to_host()
    assert P.nnz == int(meta["nnz"])
    assert np.array_equal(ip, z["indptr"]) and np.array_equal(ix, z["indices"])
    smap = fb.scatter_map_2d(P).cpu().numpy()
    assert np.array_equal(smap, z["scatter_map"])


@pytest.mark.parametrize("N,k", [(64, 1), (96, 2), (48, 3), (130, 2), (1, 1), (1, 2), (2, 3)])
def test_pattern_matches_oracle(fb, N, k):
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    for bc in ("dirichlet", "free"):
        V = fb.LagrangeSpace2D(m, k, bc=bc)
        if V.dim == 0:
            continue
        ip0, ix0 = O.from_cells(V.dim, V.cell_dofs)
        P = V.pattern()
        ip, ix = P.to_host()
        assert np.array_equal(ip, ip0) and np.array_equal(ix, ix0)
        assert np.array_equal(fb.scatter_map_2d(P).cpu().numpy(), O.scatter_map(V.cell_dofs, ip0, ix0))


def test_pattern_is_deterministic(fb):
    m = fb.rectangle_mesh(0, 0, 1, 1, 200, 200)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    a = fb.cell_pattern(V, V).to_host()
    b = fb.cell_pattern(V, V).to_host()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_pattern_of_permuted_cells(fb):
    """from_cells does not depend on the order of the cells: shuffle them, same pattern."""
    m = fb.rectangle_mesh(0, 0, 1, 1, 30, 30)
    V = fb.LagrangeSpace2D(m, 3, bc="free")
    rng = np.random.default_rng(5)
    perm = rng.permutation(m.ncells)
    import torch
    dofs = torch.as_tensor(V.cell_dofs[perm]).cuda()
    import ctypes as C
    h = C.c_void_p()
    ctx = fb.context()
    fb.lib.femd_cuda_pattern_from_cells(ctx.h, V.dim, m.ncells, V.nloc, C.c_void_p(dofs.data_ptr()), C.byref(h))
    P2 = fb.SparsityPattern(h, ctx)
    a, b = V.pattern().to_host(), P2.to_host()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_pattern_rejects_bad_dofs(fb):
    import ctypes as C
    import torch
    ctx = fb.context()
    dofs = torch.tensor([[0, 1, 7]], dtype=torch.int32).cuda()
    h = C.c_void_p()
    st = fb.lib.femd_cuda_pattern_from_cells(ctx.h, 5, 1, 3, C.c_void_p(dofs.data_ptr()), C.byref(h))
    assert st == 1 and b">= nrows" in fb.lib.femd_cuda_last_error()


def test_config2_pattern_counts(fb):
    """Config 2 (1024 x 1024, P2): the pattern the reference reports (nnz 48,136,245) and the
    oracle's, compared row by row."""
    m = fb.rectangle_mesh(0, 0, 1, 1, 1024, 1024)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    assert V.dim == 4190209
    P = V.pattern()
    assert P.nnz == 48136245
    ip, ix = P.to_host()
    ip0, ix0 = O.from_cells(V.dim, V.cell_dofs)
    assert np.array_equal(ip, ip0) and np.array_equal(ix, ix0)


def _pattern_of_cells(fb, nrows, dofs_np):
    import ctypes as C
    import torch
    dofs = torch.as_tensor(np.ascontiguousarray(dofs_np, dtype=np.int32)).cuda()
    h = C.c_void_p()
    ctx = fb.context()
    st = fb.lib.femd_cuda_pattern_from_cells(ctx.h, nrows, dofs.shape[0], dofs.shape[1], C.c_void_p(dofs.data_ptr()),
                                             C.byref(h))
    assert st == 0, fb.lib.femd_cuda_last_error()
    P = fb.SparsityPattern(h, ctx)
    P.ncells, P.nloc = dofs.shape   # what cell_pattern records for scatter_map_2d
    return P


@pytest.mark.parametrize("ncells,nloc,nrows,seed", [(5000, 6, 3000, 1), (20000, 3, 1500, 2), (600, 10, 200, 3),
                                                    (40, 6, 1000, 4)])
def test_pattern_of_random_cells(fb, ncells, nloc, nrows, seed):
    """Random cell maps with constrained (-1) entries: rows from empty to a few hundred columns,
    so both the thread-per-row path (up to 40 columns) and the warp-per-row path for the longer
    rows run; pattern, diagonal flag and scatter map against the oracle bit for bit."""
    rng = np.random.default_rng(seed)
    dofs = rng.integers(-1, nrows, size=(ncells, nloc)).astype(np.int32)
    P = _pattern_of_cells(fb, nrows, dofs)
    ip0, ix0 = O.from_cells(nrows, dofs)
    ip, ix = P.to_host()
    assert np.array_equal(ip, ip0) and np.array_equal(ix, ix0)
    lens = np.diff(ip0)
    assert lens.max() > 40 or nrows > ncells   # the long-row path ran (the last case: mostly empty rows)
    assert np.array_equal(fb.scatter_map_2d(P).cpu().numpy(), O.scatter_map(dofs, ip0, ix0))


@pytest.mark.parametrize("N,k", [(20, 4), (12, 5)])
def test_pattern_of_high_degree(fb, N, k):
    """P4 / P5: the vertex rows (61 / 91 columns on a 6-valent mesh) take the warp-per-row path,
    the edge and interior rows the thread-per-row path."""
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    V = fb.LagrangeSpace2D(m, k, bc="free")
    ip0, ix0 = O.from_cells(V.dim, V.cell_dofs)
    ip, ix = V.pattern().to_host()
    assert np.diff(ip0).max() > 40
    assert np.array_equal(ip, ip0) and np.array_equal(ix, ix0)
