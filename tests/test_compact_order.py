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


def _layout(ip, ix):
    from femd_b200 import lib
    n = ip.size - 1
    ip = np.ascontiguousarray(ip, dtype=np.int32)
    ix = np.ascontiguousarray(ix, dtype=np.int32)
    nsell, bw = C.c_longlong(), C.c_int()
    ixp = ix.ctypes.data if ix.size else None
    st = lib.femd_host_compact_layout(n, ip.ctypes.data, ixp, C.byref(nsell), C.byref(bw), None, None, None, None, None,
                                      None)
    assert st == 0, lib.femd_cuda_last_error()
    if bw.value < 0:
        return None
    ns = (n + 31) // 32
    out = dict(iperm=np.empty(max(n, 1), np.int32), rstart=np.empty(n + 1, np.int32), dst=np.empty(max(ix.size, 1), np.int32),
               off=np.empty(max(nsell.value, 1), np.int16), tlo=np.empty(max(ns, 1), np.int32),
               thi=np.empty(max(ns, 1), np.int32))
    st = lib.femd_host_compact_layout(n, ip.ctypes.data, ixp, C.byref(nsell), C.byref(bw), *[out[k].ctypes.data for k in
                                      ("iperm", "rstart", "dst", "off", "tlo", "thi")])
    assert st == 0, lib.femd_cuda_last_error()
    out.update(nsell=nsell.value, bw=bw.value, n=n, ns=ns)
    return out


@pytest.mark.parametrize("N,k", [(16, 1), (40, 2), (33, 3), (70, 2), (5, 3)])
def test_compact_layout_slices(N, k):
    """The sliced compact layout that the lockstep SpMV reads (femd_host_compact_layout, host
    code): slice widths, padding, every entry's slot and offset, and the slices' column windows,
    checked against the pattern permuted by iperm. These are the bounds the kernel relies on:
    a slot below nsell, an offset that lands in the slice's window."""
    pts, tris = O.rectangle_mesh(N)
    dofs, _, dim, _ = O.lagrange_numbering(pts.shape[0], tris, k, True)
    ip, ix = O.from_cells(dim, dofs)
    L = _layout(ip, ix)
    assert L is not None
    n, nsell, rs, off, dst = L["n"], L["nsell"], L["rstart"], L["off"][:L["nsell"]], L["dst"][:ix.size]
    iperm = L["iperm"][:n]
    assert np.array_equal(np.sort(iperm), np.arange(n))
    lens = np.diff(ip)
    klen = np.empty(n, np.int64)
    klen[iperm] = lens                                        # row lengths in the reordered order
    # slices: row k of slice t starts at the slice's base + k % 32, width = the longest row
    width = np.zeros(L["ns"], np.int64)
    for t in range(L["ns"]):
        k0, k1 = 32 * t, min(n, 32 * t + 32)
        base = rs[k0]
        assert np.array_equal(rs[k0:k1], base + np.arange(k1 - k0))
        end = rs[k1] if k1 < n else rs[n]
        assert (end - base) % 32 == 0
        width[t] = (end - base) // 32
        assert width[t] == klen[k0:k1].max()
    assert rs[n] == nsell == 32 * width.sum()
    assert nsell >= ix.size and nsell <= 1.06 * ix.size + 32 * 40   # the length sort keeps the padding small
    # every entry: its slot is row start + 32 j, j its rank by reordered column; the offset is
    # the reordered column minus the row
    rows = np.repeat(np.arange(n), lens)
    kr, kc = iperm[rows], iperm[ix]
    assert np.unique(dst).size == ix.size and dst.min() >= 0 and dst.max() < nsell
    j = (dst - rs[kr]) // 32
    assert np.array_equal((dst - rs[kr]) % 32, np.zeros_like(dst))
    assert np.all((j >= 0) & (j < klen[kr]))
    order = np.lexsort((kc, kr))
    rank = np.empty(ix.size, np.int64)
    rank[order] = np.arange(ix.size) - np.repeat(np.concatenate(([0], np.cumsum(klen)[:-1])), klen)
    assert np.array_equal(j, rank)
    assert np.array_equal(off[dst], kc - kr)
    pad = np.ones(nsell, bool)
    pad[dst] = False
    assert np.all(off[pad] == 0)
    assert L["bw"] == int(np.abs(kc - kr).max()) <= 32767
    # the slices' windows hold every column of their rows and the rows themselves
    t = kr // 32
    assert np.all(L["tlo"][t] <= kc) and np.all(L["thi"][t] >= kc)
    ks = np.arange(n)
    assert np.all(L["tlo"][ks // 32] <= ks) and np.all(L["thi"][ks // 32] >= ks)


def test_compact_layout_refuses_a_wide_pattern():
    """A star (row 0 coupled to every row) keeps a reordered bandwidth near n: over 32,767 no
    layout is made (the engine keeps the plain layout)."""
    n = 40000
    cols = [np.arange(n)] + [np.array([0, i]) for i in range(1, n)]
    ip = np.concatenate(([0], np.cumsum([c.size for c in cols]))).astype(np.int32)
    ix = np.concatenate(cols).astype(np.int32)
    assert _layout(ip, ix) is None


def test_compact_layout_rejects_bad_input():
    from femd_b200 import lib
    nsell, bw = C.c_longlong(), C.c_int()
    ip = np.array([0, 1, 2], np.int32)
    ix = np.array([0, 5], np.int32)
    st = lib.femd_host_compact_layout(2, ip.ctypes.data, ix.ctypes.data, C.byref(nsell), C.byref(bw), None, None, None,
                                      None, None, None)
    assert st == 1 and b"out of range" in lib.femd_cuda_last_error()


def test_tune_lockstep_picks_the_fastest_candidate():
    """Batch.tune_lockstep's host logic with the solve stood in for: every candidate configured
    and timed `reps` times (best of them), the fastest kept configured, ties to the first, and no
    candidates refused."""
    from femd_b200.batch import Batch
    B = object.__new__(Batch)
    B._ls_shape = dict(nnz_per_entry=16384, chunk=8, spmv="row groups", compact=True)
    cost = {8192: [3.0, 2.0], 16384: [1.5, 1.0], 32768: [1.0, 1.2], 65536: [4.0, 4.0]}
    seen, configured = [], []

    def configure_lockstep(nnz_per_entry=0, chunk=0, windows=None, compact=None):
        configured.append(nnz_per_entry)
        B._ls_shape["nnz_per_entry"] = nnz_per_entry

    def solve(bs, xs=None, *, tol, max_iter, mixed, engine):
        c = B._ls_shape["nnz_per_entry"]
        seen.append((c, max_iter, engine, tol))
        t = cost[c].pop(0)
        return None, [{"seconds": t}, {"seconds": t / 2}]

    B.configure_lockstep, B.solve = configure_lockstep, solve
    best, times = B.tune_lockstep([None], iters=7, reps=2)
    assert times == {8192: 2.0, 16384: 1.0, 32768: 1.0, 65536: 4.0}
    assert best == 16384 and configured[-1] == 16384 and B._ls_shape["nnz_per_entry"] == 16384
    assert len(seen) == 8 and all(m == 7 and e == "lockstep" and tol < 1e-200 for _, m, e, tol in seen)
    with pytest.raises(ValueError):
        B.tune_lockstep([None], candidates=())
    with pytest.raises(ValueError):
        B.tune_lockstep([None], iters=0)
