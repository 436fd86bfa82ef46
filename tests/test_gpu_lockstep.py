"""The lockstep engine of the batch (femd_cuda_batch_solve_lockstep): parity with an FP64 direct
solve and with the single FP64 solve's iteration counts, the same bits alone, in a mix and
under any table shape, and the edge cases of the stopping rule (b = 0, a converged start,
max_iter)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fb():
    import femd_b200
    return femd_b200


@pytest.fixture(scope="module")
def problems(fb):
    from femd_b200 import workloads as W
    spec = W.poisson_batch_spec(seed=11, nprob=14, nmin=4, nmax=40)
    cache = W.SpaceCache()
    return [(s, *W.build_poisson(s, cache)) for s in spec]


def direct(K, b):
    ip, ix = K.pattern.to_host()
    A = sp.csr_matrix((K.data, ix, ip), shape=(K.nrows, K.ncols))
    return spla.spsolve(A.tocsc(), b.cpu().numpy())


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("nnz_per_entry,chunk,windows", [(0, 0, True), (256, 3, True), (4096, 1, True), (0, 0, False),
                                                         (4096, 2, False)])
def test_lockstep_matches_direct_solve(fb, problems, mixed, nnz_per_entry, chunk, windows):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats)
    B.configure_lockstep(nnz_per_entry, chunk, windows)
    xs, res = B.solve(bs, tol=1e-10, mixed=mixed, engine="lockstep")
    assert B.last_status == 0
    for (s, K, b), x, r in zip(problems, xs, res):
        assert r["converged"] and not r["breakdown"] and r["status"] == 0, (s, r)
        assert r["residual"] <= 1e-9
        xd = direct(K, b)
        assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8, (s, r)
        if mixed:
            assert r["reliable_updates"] >= 1


def test_lockstep_compact_layout(fb, problems):
    """Mixed precision in the compact layout (reverse Cuthill-McKee order, 16-bit column offsets,
    the direction read from shared memory) against the plain layout and a direct solve: every
    member uses it, both layouts are within 1e-8 of the direct solution, and the compact solve
    is the same bits alone and in the mix."""
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats)
    xs, res = B.solve(bs, tol=1e-10, mixed=True, engine="lockstep")
    st = B.lockstep_stats()
    assert st["compact"] == len(mats) and st["plain"] == 0 and 0 < st["widest_window"] <= 12288
    Bp = fb.Batch(mats)
    Bp.configure_lockstep(compact=False)
    xp, resp = Bp.solve(bs, tol=1e-10, mixed=True, engine="lockstep")
    assert Bp.lockstep_stats()["compact"] == 0
    for (s, K, b), x, r, y, q in zip(problems, xs, res, xp, resp):
        assert r["converged"] and q["converged"], (s, r, q)
        xd = direct(K, b)
        for v in (x, y):
            assert np.linalg.norm(v.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8, s
    for p in (2, 9):
        xa, _ = fb.Batch([mats[p]]).solve([bs[p]], tol=1e-10, mixed=True, engine="lockstep")
        assert np.array_equal(xa[0].cpu().numpy(), xs[p].cpu().numpy())


def test_lockstep_fp64_iterations_match_the_single_solve(fb, problems):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    xs, res = fb.Batch(mats).solve(bs, tol=1e-10, mixed=False, engine="lockstep")
    for (s, K, b), x, r in zip(problems, xs, res):
        M = fb.JacobiPreconditioner(K)
        x1, conv, its, resid, brk = fb.cg_solve(K, M, b, None, 100000, 1e-10)
        assert conv and abs(its - r["iterations"]) <= 0.02 * its + 2, (s, its, r)
        x1 = x1.cpu().numpy()
        assert np.linalg.norm(x.cpu().numpy() - x1) <= 1e-8 * np.linalg.norm(x1)


@pytest.mark.parametrize("mixed", [False, True])
def test_lockstep_same_bits_alone_in_the_mix_and_any_chunk(fb, problems, mixed):
    """A member's sums are its own entry partials in entry order: the other members, the chunk
    length (when the table is compacted) and the engine's queue do not change its bits."""
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    xs, _ = fb.Batch(mats).solve(bs, tol=1e-10, mixed=mixed, engine="lockstep")
    B1 = fb.Batch(mats)
    B1.configure_lockstep(chunk=1)
    xs1, _ = B1.solve(bs, tol=1e-10, mixed=mixed, engine="lockstep")
    xs2, _ = B1.solve(bs, tol=1e-10, mixed=mixed, engine="lockstep")
    for p in range(len(mats)):
        assert np.array_equal(xs1[p].cpu().numpy(), xs[p].cpu().numpy())
        assert np.array_equal(xs2[p].cpu().numpy(), xs[p].cpu().numpy())
    for p in (0, 6, 13):
        xa, _ = fb.Batch([mats[p]]).solve([bs[p]], tol=1e-10, mixed=mixed, engine="lockstep")
        assert np.array_equal(xa[0].cpu().numpy(), xs[p].cpu().numpy())


@pytest.mark.parametrize("mixed", [False, True])
def test_lockstep_edge_cases(fb, problems, mixed):
    import torch
    (_, K0, b0), (_, K1, b1), (_, K2, b2) = problems[:3]
    xe = torch.as_tensor(direct(K1, b1)).cuda()
    B = fb.Batch([K0, K1, K2])
    bz = torch.zeros_like(b0)
    xs = [torch.ones_like(b0), xe.clone(), torch.zeros_like(b2)]
    xs, res = B.solve([bz, b1, b2], xs, tol=1e-10, max_iter=3, mixed=mixed, engine="lockstep")
    # b = 0: x = 0, converged at the start
    assert res[0]["converged"] and res[0]["iterations"] == 0 and res[0]["residual"] == 0.0
    assert not xs[0].any()
    # a start within tol: no iteration
    assert res[1]["converged"] and res[1]["iterations"] == 0
    # max_iter: stopped, not converged
    assert res[2]["iterations"] == 3 and not res[2]["converged"] and not res[2]["breakdown"]


def test_lockstep_unknown_engine_is_rejected(fb, problems):
    _, K, b = problems[0]
    with pytest.raises(ValueError):
        fb.Batch([K]).solve([b], engine="nope")


def test_pattern_batch_layout(fb, problems):
    """The compact layout built ahead of the first solve: its bandwidth (the same on a repeated
    call, which builds nothing), and a rectangular pattern refused."""
    _, K, _ = problems[-1]
    P = K.pattern
    bw = P.batch_layout()
    assert 0 < bw < P.nrows and P.batch_layout() == bw
    R = fb.SparsityPattern.from_arrays(2, 3, np.array([0, 1, 2]), np.array([0, 2]))
    with pytest.raises(ValueError, match="square"):
        R.batch_layout()


def test_tune_lockstep(fb, problems):
    """The lockstep autotuner: each candidate entry size timed on the members, the fastest kept
    configured, and a solve with it within 1e-8 of the direct solutions."""
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats)
    best, times = B.tune_lockstep(bs, candidates=(2048, 8192), iters=6, reps=1)
    assert set(times) == {2048, 8192} and all(t > 0 for t in times.values())
    assert best in times and times[best] == min(times.values())
    assert B._ls_shape["nnz_per_entry"] == best
    xs, res = B.solve(bs, tol=1e-10, mixed=True, engine="lockstep")
    for (s, K, b), x, r in zip(problems, xs, res):
        assert r["converged"], (s, r)
        xd = direct(K, b)
        assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8, (s, r)
    with pytest.raises(ValueError):
        B.tune_lockstep(bs, candidates=())
