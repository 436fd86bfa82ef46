"""Host setup of the boundary terms (no GPU): the exterior facet list with side markers, the facet
rule (Gauss-Legendre points per local edge and the tabulation there) and the raw numbering,
against the reference's fixtures."""
import numpy as np
import pytest

from conftest import DS_CASES, GOLDEN_CASES, golden


@pytest.mark.parametrize("name", DS_CASES)
def test_facet_list_and_rule(name):
    import femd_b200 as fb
    from femd_b200.lift import SIDES
    z, meta = golden(name)
    N, k = int(meta["N"]), int(meta["k"])
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    cell = np.empty(3 * m.ncells, dtype=np.int32)
    local, marker = np.empty_like(cell), np.empty_like(cell)
    mk = np.array(SIDES, dtype=np.int32)
    nf = fb.lib.femd_host_exterior_facets(m.nverts, m.ncells, m.tris.ctypes.data, m.points.ctypes.data, 0.0, 0.0, 1.0, 1.0,
                                          mk.ctypes.data, cell.ctypes.data, local.ctypes.data, marker.ctypes.data)
    assert nf == 4 * N
    assert np.array_equal(cell[:nf], z["facet_cell"]) and np.array_equal(local[:nf], z["facet_local"])
    assert np.array_equal(marker[:nf], z["facet_marker"])
    nl = (k + 1) * (k + 2) // 2
    xi, eta, gw, ref = np.empty(192), np.empty(192), np.empty(64), np.empty(3 * 64 * 3 * nl)
    nq = fb.lib.femd_host_facet_rule(k, 2 * k, xi.ctypes.data, eta.ctypes.data, gw.ctypes.data, ref.ctypes.data)
    assert nq == int(meta["facet_nq"])
    assert np.all(np.abs(ref[:3 * nq * 3 * nl] - z["facet_ref"]) <= 1e-13)
    assert abs(gw[:nq].sum() - 2.0) <= 1e-14


@pytest.mark.parametrize("name", [n for n in GOLDEN_CASES if "heat" not in n][:6] + DS_CASES)
def test_raw_numbering(name):
    import ctypes as C

    import femd_b200 as fb
    z, meta = golden(name)
    N, k = int(meta["N"]), int(meta["k"])
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    nl = (k + 1) * (k + 2) // 2
    raw = np.empty((m.ncells, nl), dtype=np.int32)
    rd = C.c_int()
    assert fb.lib.femd_host_lagrange_raw(m.nverts, m.ncells, m.tris.ctypes.data, k, raw.ctypes.data, C.byref(rd)) == 0
    assert np.array_equal(raw.reshape(-1), z["cell_raw_dofs"]) and rd.value == int(meta["raw_dim"])


def test_lagrange_nodes():
    import femd_b200 as fb
    xi, eta = np.empty(10), np.empty(10)
    assert fb.lib.femd_host_lagrange_nodes(3, xi.ctypes.data, eta.ctypes.data) == 10
    assert np.allclose(xi[:3], [0, 1, 0]) and np.allclose(eta[:3], [0, 0, 1])
    assert np.allclose([xi[9], eta[9]], [1 / 3, 1 / 3])
