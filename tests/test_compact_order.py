"""The ordering of the batched engine's compact layout (femd_host_rcm_order, host code): a
permutation, deterministic, and a bandwidth as small as scipy's reverse Cuthill-McKee gives on
the config-4 patterns (P1-P3 on rectangle meshes, whose own numbering puts edge and interior
nodes far from the vertices), small enough for 16-bit column offsets."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sps
from scipy.sparse.csgraph import reverse_cuthill_mckee

from oracle import oracle as O


def _order(ip, ix):
    from femd_b200 import lib
    n = ip.size - 1
    out = np.empty(max(n, 1), dtype=np.int32)
    ip = np.ascontiguousarray(ip, dtype=np.int32)
    ix = np.ascontiguousarray(ix, dtype=np.int32)
    st = lib.femd_host_rcm_order(n, ip.ctypes.data, ix.ctypes.data if ix.size else None, out.ctypes.data)
    assert st == 0, lib.femd_cuda_last_error()
    return out[:n]


def _bandwidth(ip, ix, order):
    n = ip.size - 1
    A = sps.csr_matrix((np.ones(ix.size), ix, ip), shape=(n, n))[order][:, order].tocoo()
    return int(np.abs(A.row - A.col).max())


@pytest.mark.parametrize("N,k", [(16, 1), (40, 2), (33, 3), (90, 2)])
def test_rcm_bandwidth(N, k):
    pts, tris = O.rectangle_mesh(N)
    dofs, _, dim, _ = O.lagrange_numbering(pts.shape[0], tris, k, True)
    ip, ix = O.from_cells(dim, dofs)
    order = _order(ip, ix)
    assert np.array_equal(np.sort(order), np.arange(dim))
    assert np.array_equal(order, _order(ip, ix))
    bw = _bandwidth(ip, ix, order)
    ref = _bandwidth(ip, ix, reverse_cuthill_mckee(sps.csr_matrix((np.ones(ix.size), ix, ip), shape=(dim, dim)),
                                                   symmetric_mode=True))
    rows = np.repeat(np.arange(dim), np.diff(ip))
    assert bw <= 1.25 * ref + 2 and bw < 32768
    assert bw < np.abs(ix - rows).max() or N <= 16


def test_rcm_disconnected_and_edge_cases():
    # two components, an isolated node and an empty pattern
    ip = np.array([0, 2, 4, 5, 7, 9, 9])
    ix = np.array([0, 1, 0, 1, 2, 3, 4, 3, 4])
    order = _order(ip, ix)
    assert np.array_equal(np.sort(order), np.arange(6))
    assert _order(np.array([0]), np.array([], dtype=np.int32)).size == 0
    from femd_b200 import lib
    bad = np.array([0, 1], dtype=np.int32)
    assert lib.femd_host_rcm_order(1, bad.ctypes.data, np.array([3], dtype=np.int32).ctypes.data,
                                   np.empty(1, dtype=np.int32).ctypes.data) == 1
