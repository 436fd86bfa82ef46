"""CPU checks of the C ABI: the library loads, exports every entry point include/femd_cuda.h
declares, and its host-side setup (mesh, numbering, quadrature, tabulation) agrees with the
oracle bit for bit.  No GPU work is started here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

LIB = os.path.join(ROOT, "femd_b200", "libfemd_cuda.so")
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        names |= set(re.findall(r"FEMD_API\s+[^;(]*?\b(femd_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first (python -m femd_b200.build)"
    names = declared()
    assert len(names) >= 30
    lib = C.CDLL(LIB)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (femd_\w+)", out))
    assert set(names) <= exported


def test_python_binding_covers_every_symbol():
    from femd_b200 import _native as N
    assert set(declared()) == set(N.SIGNATURES)


def test_version_and_error_text():
    from femd_b200 import lib
    assert lib.femd_cuda_version().decode().startswith("femd_b200")
    # a host-side call with a bad argument sets the thread's error text
    pts = np.empty((4, 2))
    tris = np.empty((2, 3), dtype=np.int32)
    st = lib.femd_host_rectangle_mesh(1.0, 0.0, 0.0, 1.0, 1, 1, pts.ctypes.data, tris.ctypes.data)
    assert st == 1
    assert "x1 > x0" in lib.femd_cuda_last_error().decode()


@pytest.mark.parametrize("N,k", [(1, 1), (2, 2), (3, 3), (7, 1), (8, 2), (5, 3), (4, 4), (3, 5), (40, 2), (33, 3)])
def test_host_numbering_matches_oracle(N, k):
    import femd_b200 as fb
    m = fb.rectangle_mesh(0, 0, 1, 1, N, N)
    pts, tris = O.rectangle_mesh(N)
    assert np.array_equal(m.points, pts) and np.array_equal(m.tris, tris)
    for bc in ("dirichlet", "free"):
        V = fb.LagrangeSpace2D(m, k, bc=bc)
        dofs, raw, dim, raw_dim = O.lagrange_numbering(pts.shape[0], tris, k, bc == "dirichlet")
        assert V.dim == dim and V.raw_dim == raw_dim
        assert np.array_equal(V.cell_dofs, dofs)


def test_host_numbering_nonsquare_rectangle():
    import femd_b200 as fb
    m = fb.rectangle_mesh(-1.0, 0.5, 2.0, 1.0, 7, 3)
    V = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    assert V.dim == (2 * 7 - 1) * (2 * 3 - 1)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 6])
def test_host_quadrature_and_tabulation(k):
    import femd_b200 as fb
    m = fb.rectangle_mesh(0, 0, 1, 1, 2, 2)
    V = fb.LagrangeSpace2D(m, k)
    for deg in range(0, 14):      # degree 13: 7 x 8 = 56 points; the tables hold at most 64
        Q = fb.Cache2D(V, deg)
        xi, eta, w = O.triangle_quadrature(deg)
        assert np.array_equal(Q.xi, xi) and np.array_equal(Q.eta, eta) and np.array_equal(Q.w, w)
        assert np.array_equal(Q.ref, O.tabulate(k, xi, eta))
    # the basis is nodal and a partition of unity
    Q = fb.Cache2D(V, 4)
    assert np.allclose(Q.ref[:, 0, :].sum(axis=1), 1.0, atol=1e-13)
    assert np.allclose(Q.ref[:, 1, :].sum(axis=1), 0.0, atol=1e-11)


def test_host_errors():
    import femd_b200 as fb
    with pytest.raises(ValueError):
        fb.rectangle_mesh(0, 0, 1, 1, 0, 3)
    m = fb.rectangle_mesh(0, 0, 1, 1, 2, 2)
    with pytest.raises(ValueError):
        fb.LagrangeSpace2D(m, 0)
    with pytest.raises(ValueError):
        fb.LagrangeSpace2D(m, 2, bc="periodic")
