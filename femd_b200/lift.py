"""Boundary terms on the GPU: ds(marker) integrals on exterior facets and the Dirichlet lift.

    FacetCache2D            cache_2d.hpp:126-184         exterior facets (all, or by marker), their
                                                          Gauss-Legendre rule, per-point geometry
    assemble_facet_matrix   assembly_2d.hpp:219-305      K += the ds terms (Robin)
    assemble_facet_vector   assembly_2d.hpp:173-211      f += the ds terms (Neumann / Robin data)
    lift(V, g)              spaces2d.py:373-414          u_g on V.unconstrained: g at the eliminated nodes
    Lift.action(a)          forms.py:2892 + linalg.py:753  a(u_g, v), assembled on the device
    Lift.compose(x)         spaces2d.py:376              u = V.prolongate(x) + u_g (raw numbering)

The facet list and the rule are host setup (the reference builds them on the host too); the
per-point geometry, the coefficient programs and the assembly run in libfemd_cuda.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .core import Coef, LagrangeSpace2D, _Handle, _np_ptr, _torch, assemble_vector_2d, check, context, lib

SIDES = (1, 2, 3, 4)        # rectangle_mesh's side markers: bottom, right, top, left (structured.hpp:26-31)


class FacetCache2D:
    """The exterior facets of V's mesh whose marker is in markers (all when None), with the
    Gauss-Legendre rule exact to `degree` along each edge (Cache2D(V, degree, markers, all))."""

    def __init__(self, V: LagrangeSpace2D, degree: int, markers=None, ctx=None):
        self.space, self.degree = V, int(degree)
        self.ctx = ctx or context()
        m = V.mesh
        x0, y0 = m.points.min(axis=0)
        x1, y1 = m.points.max(axis=0)
        cell = np.empty(3 * m.ncells, dtype=np.int32)
        local = np.empty_like(cell)
        marker = np.empty_like(cell)
        mk = np.array(SIDES, dtype=np.int32)
        nf = lib.femd_host_exterior_facets(m.nverts, m.ncells, _np_ptr(m.tris), _np_ptr(m.points), float(x0), float(y0),
                                           float(x1), float(y1), _np_ptr(mk), _np_ptr(cell), _np_ptr(local),
                                           _np_ptr(marker))
        if nf < 0:
            check(-nf)
        keep = np.ones(nf, dtype=bool) if markers is None else np.isin(marker[:nf], np.asarray(list(markers)))
        self.cell = np.ascontiguousarray(cell[:nf][keep])
        self.local = np.ascontiguousarray(local[:nf][keep])
        self.marker = np.ascontiguousarray(marker[:nf][keep])
        nl = V.nloc
        xi, eta, gw = np.empty(3 * 64), np.empty(3 * 64), np.empty(64)
        ref = np.empty(3 * 64 * 3 * nl)
        nq = lib.femd_host_facet_rule(V.degree, self.degree, _np_ptr(xi), _np_ptr(eta), _np_ptr(gw), _np_ptr(ref))
        if nq < 0:
            check(-nq)
        self.xi, self.eta, self.gw = xi[:3 * nq].copy(), eta[:3 * nq].copy(), gw[:nq].copy()
        self.ref = ref[:3 * nq * 3 * nl].reshape(3, nq, 3, nl).copy()
        h = C.c_void_p()
        P = V.pattern(self.ctx)
        check(lib.femd_cuda_facets_create(self.ctx.h, P.h, self.nent, _np_ptr(self.cell), _np_ptr(self.local), C.byref(h)))
        self._h = _Handle(h)
        self._pts = None

    @property
    def h(self):
        return self._h.h

    @property
    def nent(self):
        return int(self.cell.size)

    @property
    def nq(self):
        return int(self.gw.size)

    def c_rule(self):
        V = self.space
        return N.femd_facet_rule(V.degree, V.nloc, self.nq, self.xi.ctypes.data, self.eta.ctypes.data, self.gw.ctypes.data,
                                 self.ref.ctypes.data)

    def points(self):
        """(x, y, w, nx, ny) at the facet points [f nq + q], float64 device tensors (computed once)."""
        if self._pts is None:
            torch = _torch()
            n = self.nent * self.nq
            out = [torch.empty(n, dtype=torch.float64, device=f"cuda:{self.ctx.device}") for _ in range(5)]
            mesh = self.space.mesh.c_struct(self.ctx)
            rule = self.c_rule()
            self.ctx.enter()
            st = lib.femd_cuda_facet_points(self.ctx.h, self.h, C.byref(mesh), C.byref(rule),
                                            *[C.c_void_p(t.data_ptr()) for t in out])
            self.ctx.leave()
            check(st)
            self._pts = tuple(out)
        return self._pts


def _facet_coefs(coeffs):
    out = [c if isinstance(c, Coef) else Coef.const(c) for c in coeffs]
    return out, (N.femd_coef * len(out))(*[c.c_struct() for c in out])


def assemble_facet_matrix(F: FacetCache2D, a, b, coeffs, K):
    """K += sum_t integral over F's facets of c_t (D^a_t phi_i)(D^b_t phi_j) ds; each coefficient a
    number or Coef.points(values at the facet points)."""
    if len(a) != len(b) or len(a) != len(coeffs):
        raise ValueError("assembly_2d: one coefficient array per term")
    keep, carr = _facet_coefs(coeffs)
    mesh = F.space.mesh.c_struct(F.ctx)
    rule = F.c_rule()
    ai, bi = (C.c_int * len(a))(*a), (C.c_int * len(b))(*b)
    F.ctx.enter()
    st = lib.femd_cuda_assemble_facet_matrix(F.ctx.h, F.h, C.byref(mesh), C.byref(rule), len(a), ai, bi, carr, K.h)
    F.ctx.leave()
    check(st)
    del keep
    return K


def assemble_facet_vector(F: FacetCache2D, a, coeffs, f):
    """f += sum_t integral over F's facets of c_t D^a_t phi_i ds (f a float64 device tensor)."""
    if len(a) != len(coeffs):
        raise ValueError("assembly_2d: one coefficient array per term")
    keep, carr = _facet_coefs(coeffs)
    mesh = F.space.mesh.c_struct(F.ctx)
    rule = F.c_rule()
    ai = (C.c_int * len(a))(*a)
    F.ctx.enter()
    st = lib.femd_cuda_assemble_facet_vector(F.ctx.h, F.h, C.byref(mesh), C.byref(rule), len(a), ai, carr,
                                             C.c_void_p(f.data_ptr()))
    F.ctx.leave()
    check(st)
    del keep
    return f


# ---- the raw numbering and the lift ------------------------------------------------------------
def raw_numbering(V: LagrangeSpace2D):
    """(cell_raw ncells x nloc, raw_dim, raw_of): the numbering of V.unconstrained and, for every
    dof of V, its raw node (cached on the space)."""
    r = getattr(V, "_raw", None)
    if r is None:
        m = V.mesh
        cell_raw = np.empty((m.ncells, V.nloc), dtype=np.int32)
        rd = C.c_int()
        check(lib.femd_host_lagrange_raw(m.nverts, m.ncells, _np_ptr(m.tris), V.degree, _np_ptr(cell_raw), C.byref(rd)))
        raw_of = np.full(V.dim, -1, dtype=np.int64)
        cd = V.cell_dofs.reshape(-1)
        sel = cd >= 0
        raw_of[cd[sel]] = cell_raw.reshape(-1)[sel]
        r = V._raw = (cell_raw, rd.value, raw_of.astype(np.int32))
    return r


def raw_coordinates(V: LagrangeSpace2D):
    """(raw_dim, 2) coordinates of every node of V.unconstrained: each cell maps its local nodes
    (x = P0 + J (xi, eta))."""
    cell_raw, rd, _ = raw_numbering(V)
    k, nl = V.degree, V.nloc
    xi, eta = np.empty(nl), np.empty(nl)
    lib.femd_host_lagrange_nodes(k, _np_ptr(xi), _np_ptr(eta))
    P, T = V.mesh.points, V.mesh.tris
    p0, p1, p2 = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    xy = p0[:, None, :] + xi[None, :, None] * (p1 - p0)[:, None, :] + eta[None, :, None] * (p2 - p0)[:, None, :]
    out = np.empty((rd, 2))
    out[cell_raw.reshape(-1)] = xy.reshape(-1, 2)
    return out


def _values(g, xy):
    if callable(g):
        return np.broadcast_to(np.asarray(g(xy[:, 0], xy[:, 1]), dtype=np.float64), (xy.shape[0],)).copy()
    return np.full(xy.shape[0], float(g))


class Lift:
    """u_g: a vector of V.unconstrained (raw numbering, float64 on the device) that carries the
    Dirichlet data on the eliminated nodes and zero elsewhere."""

    def __init__(self, V: LagrangeSpace2D, raw):
        self.space = V
        self.vector = raw

    def action(self, a):
        """a(u_g, v) for the test functions of V (the load a.action(u_g).assemble() that fd.solve
        takes off b): per term, the coefficient times D^b u_g at the points of a's rule, assembled
        as a vector on the device."""
        from .forms import MUL, INPUT, Integrand, eval_field
        torch = _torch()
        V = self.space
        cell_raw, _, _ = raw_numbering(V)
        ctx = a.V.pattern().ctx
        dev = f"cuda:{ctx.device}"
        raw_dofs = torch.as_tensor(cell_raw).to(dev)
        prod = Integrand([[INPUT, 0, 0, 0], [INPUT, 1, 1, 0], [MUL, 0, 0, 1]], 2, 0, 2)
        A = a.A
        vals = A._values(a.vectors, ctx)
        f = torch.zeros(V.dim, dtype=torch.float64, device=dev)
        for G in A.groups:
            if not G["terms"]:
                continue
            Q = G["QT"]
            du = eval_field(Q, self.vector, [0, 1, 2], raw_dofs=raw_dofs, ctx=ctx)
            np_ = V.mesh.ncells * Q.nq
            coefs, codes = [], []
            for prog, inputs, cidx, ta, tb in G["terms"]:
                cv = [a.consts[k] for k in cidx]
                ct = prog.evaluate_cells(Q, [vals[i] for i in inputs], cv, ctx=ctx)
                coefs.append(Coef.points(prod.evaluate(np_, [ct, du[tb * np_:(tb + 1) * np_]], [], ctx=ctx)))
                codes.append(ta)
            f += assemble_vector_2d(Q, codes, coefs)
        return f

    def compose(self, x):
        """u = V.prolongate(x) + u_g on the raw numbering (a new device tensor)."""
        torch = _torch()
        V = self.space
        _, rd, raw_of = raw_numbering(V)
        ctx = context()
        u = self.vector.clone()
        ro = torch.as_tensor(raw_of).to(u.device)
        ctx.enter()
        st = lib.femd_cuda_prolongate(ctx.h, V.dim, C.c_void_p(ro.data_ptr()), C.c_void_p(x.data_ptr()),
                                      C.c_void_p(u.data_ptr()))
        ctx.leave()
        check(st)
        return u


def lift(V: LagrangeSpace2D, g):
    """V.lift(g): g a number, a callable g(x, y) (vectorized) or a dict {marker: number or
    callable}; the data at the eliminated nodes of V (every exterior side on this path), zero
    elsewhere.  Where two sides with different data meet, the corner takes the data of the larger
    marker."""
    torch = _torch()
    _, rd, raw_of = raw_numbering(V)
    raw = np.zeros(rd)
    cons = np.setdiff1d(np.arange(rd), raw_of)
    if V.bc != "dirichlet" or cons.size == 0:
        if g is not None and not (isinstance(g, (int, float)) and g == 0):
            raise ValueError("lift(): this space has no Dirichlet condition built in; natural data enter through "
                             "ds(marker)")
        return Lift(V, torch.as_tensor(raw).cuda())
    xy = raw_coordinates(V)
    if isinstance(g, dict):
        for mkr in sorted(g):
            if int(mkr) not in SIDES:
                raise ValueError(f"lift(): marker {mkr} carries no Dirichlet condition in this space (Dirichlet "
                                 f"markers {list(SIDES)}); natural data enter through ds({mkr})")
            nodes = _side_nodes(V, int(mkr), xy)
            nodes = nodes[np.isin(nodes, cons)]
            raw[nodes] = _values(g[mkr], xy[nodes])
    elif g is not None:
        raw[cons] = _values(g, xy[cons])
    return Lift(V, torch.as_tensor(raw).cuda())


def _side_nodes(V, marker, xy):
    """The raw nodes on side `marker` of the rectangle (its facets' nodes)."""
    x0, y0 = V.mesh.points.min(axis=0)
    x1, y1 = V.mesh.points.max(axis=0)
    sel = {1: xy[:, 1] == y0, 2: xy[:, 0] == x1, 3: xy[:, 1] == y1, 4: xy[:, 0] == x0}[marker]
    return np.nonzero(sel)[0]
