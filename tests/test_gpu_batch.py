"""K7, the batched persistent PCG: parity with an FP64 direct solve, the same bits alone and in
a mix, multi-block teams, and failure detection (a team barrier that runs out, a host abort)
without faulting the GPU."""
import threading
import time

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
    spec = W.poisson_batch_spec(seed=7, nprob=12, nmin=4, nmax=24)
    cache = W.SpaceCache()
    out = []
    for s in spec:
        K, b = W.build_poisson(s, cache)
        out.append((s, K, b))
    return out


def direct(K, b):
    ip, ix = K.pattern.to_host()
    A = sp.csr_matrix((K.data, ix, ip), shape=(K.nrows, K.ncols))
    return spla.spsolve(A.tocsc(), b.cpu().numpy())


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_matches_direct_solve(fb, problems, mixed):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats)
    xs, res = B.solve(bs, tol=1e-10, mixed=mixed)
    assert B.last_status == 0
    for (s, K, b), x, r in zip(problems, xs, res):
        assert r["converged"] and not r["breakdown"], (s, r)
        assert r["residual"] <= 1e-9
        xd = direct(K, b)
        assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8, (s, r)
        if mixed:
            assert r["reliable_updates"] >= 1


def test_batch_fp64_matches_single_solve_iterations(fb, problems):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    xs, res = fb.Batch(mats).solve(bs, tol=1e-10, mixed=False)
    for (s, K, b), r in zip(problems, res):
        M = fb.JacobiPreconditioner(K)
        _, conv, its, resid, brk = fb.cg_solve(K, M, b, None, 100000, 1e-10)
        assert conv and abs(its - r["iterations"]) <= 0.02 * its + 2


@pytest.mark.parametrize("mixed", [False, True])
def test_same_bits_alone_and_in_the_mix(fb, problems, mixed):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    xs, _ = fb.Batch(mats).solve(bs, tol=1e-10, mixed=mixed)
    for p in (0, 5, 11):
        xa, _ = fb.Batch([mats[p]]).solve([bs[p]], tol=1e-10, mixed=mixed)
        assert np.array_equal(xa[0].cpu().numpy(), xs[p].cpu().numpy())


@pytest.mark.parametrize("mixed", [False, True])
def test_multi_block_teams(fb, problems, mixed):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats, nnz_per_block=256)          # small blocks: teams of several blocks
    info = B.info()
    assert info["teams"].max() > 1
    xs, res = B.solve(bs, tol=1e-10, mixed=mixed)
    assert B.last_status == 0
    for (s, K, b), x, r in zip(problems, xs, res):
        assert r["converged"]
        xd = direct(K, b)
        assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8
    # repeated solve: the same bits (deterministic team reductions)
    xs2, _ = B.solve(bs, tol=1e-10, mixed=mixed)
    for x, x2 in zip(xs, xs2):
        assert np.array_equal(x.cpu().numpy(), x2.cpu().numpy())


def test_team_barrier_timeout_is_reported_and_the_context_survives(fb, problems):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats, nnz_per_block=256)
    teams = B.info()["teams"]
    ghost = int(np.argmax(teams))
    B.debug(ghost_problem=ghost, spin_limit=1 << 14)     # one member that never comes; short waits
    t0 = time.time()
    _, res = B.solve(bs, tol=1e-10)
    assert B.last_status == 6                             # FEMD_ETIMEOUT
    assert any(r["status"] == 6 for r in res)
    assert time.time() - t0 < 30
    B.debug(ghost_problem=-1, spin_limit=0)
    xs, res = B.solve(bs, tol=1e-10)
    assert B.last_status == 0 and all(r["converged"] for r in res)


def test_host_abort(fb):
    from femd_b200 import workloads as W
    cache = W.SpaceCache()
    K, b = W.build_poisson(dict(N=160, k=2, c=1.0, seed=3), cache)
    B = fb.Batch([K], nnz_per_block=1 << 16)
    out = {}

    def run():
        out["x"], out["res"] = B.solve([b], tol=1e-300, max_iter=200_000, mixed=False)

    th = threading.Thread(target=run)
    th.start()
    time.sleep(0.5)
    B.abort()
    th.join(timeout=60)
    assert not th.is_alive()
    assert B.last_status == 7                             # FEMD_EABORT
    assert out["res"][0]["status"] == 7
