"""Device dof numbering (femd_cuda_lagrange_numbering) against the host numbering, which the
oracle pins to the reference (tests/test_oracle_pins.py): the same cell -> dof map, dimension
and raw dimension, bit for bit, on structured and scrambled meshes, and the same errors."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


def same(fb, m, k, bc):
    Vh = fb.LagrangeSpace2D(m, k, bc=bc)
    Vd = fb.LagrangeSpace2D(m, k, bc=bc, numbering="device")
    assert (Vd.dim, Vd.raw_dim) == (Vh.dim, Vh.raw_dim)
    assert np.array_equal(Vd.cell_dofs, Vh.cell_dofs)
    assert np.array_equal(Vd.cell_dofs_device().cpu().numpy(), Vh.cell_dofs)
    return Vh, Vd


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("bc", ["free", "dirichlet"])
@pytest.mark.parametrize("nx,ny", [(1, 1), (3, 2), (17, 9), (64, 64)])
def test_device_numbering_equals_host(fb, nx, ny, k, bc):
    same(fb, fb.rectangle_mesh(0, 0, 1, 1, nx, ny), k, bc)


@pytest.mark.parametrize("k", [1, 2, 3])
def test_device_numbering_on_a_scrambled_mesh(fb, k):
    """Cells in random order, vertices relabelled, each triangle's vertices rotated: the
    first-encounter order and the edge directions change, the two numberings still agree."""
    m = fb.rectangle_mesh(0, 0, 1, 1, 40, 30)
    rng = np.random.default_rng(3)
    perm_v = rng.permutation(m.nverts)
    tris = perm_v[m.tris][rng.permutation(m.ncells)]
    rot = rng.integers(0, 3, len(tris))
    tris = np.stack([np.roll(t, r) for t, r in zip(tris, rot)]).astype(np.int32)
    pts = np.empty_like(m.points)
    pts[perm_v] = m.points
    for bc in ("free", "dirichlet"):
        same(fb, fb.Mesh2D(pts, tris), k, bc)


def test_device_numbering_at_the_config2_size(fb):
    m = fb.rectangle_mesh(0, 0, 1, 1, 640, 640)
    t0 = time.perf_counter()
    Vh = fb.LagrangeSpace2D(m, 2, bc="dirichlet")
    th = time.perf_counter() - t0
    fb.LagrangeSpace2D(m, 2, bc="dirichlet", numbering="device")          # warm-up
    t0 = time.perf_counter()
    Vd = fb.LagrangeSpace2D(m, 2, bc="dirichlet", numbering="device")
    td = time.perf_counter() - t0
    assert Vd.dim == Vh.dim and np.array_equal(Vd.cell_dofs, Vh.cell_dofs)
    print(f"640 x 640 P2 numbering: host {th * 1e3:.1f} ms, device {td * 1e3:.1f} ms (with the copy back)")


def test_device_numbering_errors(fb):
    pts = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [-1, -1]], dtype=np.float64)
    fan = np.array([[0, 1, 2], [1, 3, 2], [2, 4, 1]], dtype=np.int32)     # edge (1, 2) in three triangles
    for numbering in ("host", "device"):
        with pytest.raises(ValueError, match="more than two triangles"):
            fb.LagrangeSpace2D(fb.Mesh2D(pts, fan), 2, numbering=numbering)
    bad = np.array([[0, 1, 7]], dtype=np.int32)
    for numbering in ("host", "device"):
        with pytest.raises(ValueError, match="out of range"):
            fb.LagrangeSpace2D(fb.Mesh2D(pts, bad), 2, numbering=numbering)
    with pytest.raises(ValueError):
        fb.LagrangeSpace2D(fb.rectangle_mesh(0, 0, 1, 1, 2, 2), 2, numbering="gpu")
