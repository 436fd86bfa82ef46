"""The device numbering's algorithm (csrc/numbering.cu), restated step by step in numpy, gives
the host numbering's map (femd_host_lagrange_numbering, pinned to the reference): half-edges
counted into a bucket per smaller vertex, each bucket sorted by (larger vertex, half-edge),
first appearances ranked by a scan, exterior nodes eliminated, the rest renumbered by a scan.
No GPU: this checks the order of operations the kernels implement."""
import ctypes as C

import numpy as np
import pytest


def bucket_numbering(nverts, tris, k, all_exterior):
    ncells = len(tris)
    nh = 3 * ncells
    de, nint, nloc = k - 1, (k - 1) * (k - 2) // 2, (k + 1) * (k + 2) // 2
    t = np.arange(nh)
    c, i = t // 3, t % 3
    a = tris[c, (i + 1) % 3]
    b = tris[c, (i + 2) % 3]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    cnt = np.bincount(lo, minlength=nverts)                       # k_half_count
    bptr = np.concatenate([[0], np.cumsum(cnt)])                  # exclusive scan
    first = np.zeros(nh, dtype=np.int64)
    cell_edge = np.empty(nh, dtype=np.int64)
    exterior = np.empty(nh, dtype=bool)
    buckets = []
    for v in range(nverts):                                       # k_half_fill + k_bucket_sort
        mem = np.nonzero(lo == v)[0]
        mem = mem[np.lexsort((mem, hi[mem]))]                     # (larger vertex, half-edge)
        assert len(mem) == bptr[v + 1] - bptr[v]
        p = 0
        while p < len(mem):
            e = p + 1
            while e < len(mem) and hi[mem[e]] == hi[mem[p]]:
                e += 1
            assert e - p <= 2
            first[mem[p]] = 1
            buckets.append(mem[p:e])
            p = e
    rank = np.cumsum(first) - first                               # exclusive scan
    for seg in buckets:                                           # k_bucket_edges
        cell_edge[seg] = rank[seg[0]]
        exterior[seg] = len(seg) == 1
    nedges = int(rank[-1] + first[-1])
    voff = nverts
    rd = voff + nedges * de + ncells * nint
    keep = np.ones(rd, dtype=np.int64)
    if all_exterior:                                              # k_eliminate
        for h in np.nonzero(exterior)[0]:
            keep[a[h]] = keep[b[h]] = 0
            keep[voff + cell_edge[h] * de + np.arange(de)] = 0
    r2a = np.cumsum(keep) - keep                                  # exclusive scan
    out = np.empty((ncells, nloc), dtype=np.int64)                # k_cell_dofs
    for cc in range(ncells):
        raw = list(tris[cc])
        for ii in range(3):
            g = cell_edge[3 * cc + ii]
            flip = tris[cc, (ii + 1) % 3] > tris[cc, (ii + 2) % 3]
            raw += [voff + g * de + (de - 1 - j if flip else j) for j in range(de)]
        raw += [voff + nedges * de + cc * nint + j for j in range(nint)]
        raw = np.array(raw)
        out[cc] = np.where(keep[raw] == 1, r2a[raw], -1)
    return out, int(r2a[-1] + keep[-1]), rd


def host_numbering(nverts, tris, k, all_exterior):
    from femd_b200 import _native as N
    nloc = (k + 1) * (k + 2) // 2
    tris = np.ascontiguousarray(tris, dtype=np.int32)
    out = np.empty((len(tris), nloc), dtype=np.int32)
    dim, raw = C.c_int(), C.c_int()
    st = N.lib.femd_host_lagrange_numbering(nverts, len(tris), tris.ctypes.data, k, int(all_exterior), out.ctypes.data,
                                            C.byref(dim), C.byref(raw))
    assert st == 0
    return out, dim.value, raw.value


def rect_tris(nx, ny):
    W = nx + 1
    out = []
    for j in range(ny):
        for i in range(nx):
            a = j * W + i
            out += [[a, a + 1, a + W + 1], [a, a + W + 1, a + W]]
    return (nx + 1) * (ny + 1), np.array(out, dtype=np.int64)


@pytest.mark.parametrize("k", [1, 2, 3, 4])
@pytest.mark.parametrize("all_exterior", [False, True])
@pytest.mark.parametrize("scramble", [False, True])
def test_bucket_algorithm_equals_host(k, all_exterior, scramble):
    nverts, tris = rect_tris(7, 5)
    if scramble:
        rng = np.random.default_rng(k)
        perm_v = rng.permutation(nverts)
        tris = perm_v[tris][rng.permutation(len(tris))]
        tris = np.stack([np.roll(t, r) for t, r in zip(tris, rng.integers(0, 3, len(tris)))])
    got, dim, rd = bucket_numbering(nverts, tris, k, all_exterior)
    ref, rdim, rrd = host_numbering(nverts, tris, k, all_exterior)
    assert (dim, rd) == (rdim, rrd)
    assert np.array_equal(got, ref)
