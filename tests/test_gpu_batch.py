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


def test_launch_shapes_and_autotuner(fb, problems):
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    B = fb.Batch(mats)
    for block, npb, npt in ((128, 1024, 2), (512, 4096, 2), (256, 8192, 4), (128, 2048, 8)):
        B.configure(block, npb, npt)
        xs, res = B.solve(bs, tol=1e-10, mixed=True)
        assert B.last_status == 0 and B.params()["block"] == block
        assert B.params()["graph"] in (1, -1)
        for (s, K, b), x, r in zip(problems, xs, res):
            assert r["converged"]
            xd = direct(K, b)
            assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8
    p, sec = B.tune(bs, max_iter=20, mixed=True)
    assert p["block"] in (128, 256, 512) and p["nnz_per_thread"] in (2, 4, 8) and sec > 0
    assert p["nnz_per_block"] in (8192, 16384, 32768, 65536, 131072)
    xs, res = B.solve(bs, tol=1e-10, mixed=True)
    assert all(r["converged"] for r in res)


@pytest.mark.parametrize("mixed", [False, True])
def test_resumable_steps_give_the_same_bits(fb, problems, mixed):
    """Stepping a few iterations per launch, with members joining part-way through, gives the
    bits of one launch per member."""
    import torch
    mats = [K for _, K, _ in problems]
    bs = [b for _, _, b in problems]
    xs_ref, res_ref = fb.Batch(mats).solve(bs, tol=1e-10, mixed=mixed)
    B = fb.Batch()
    ids, xs = [], []
    done = {}
    for p in range(len(mats)):
        i = B.add(mats[p])
        ids.append(i)
        xs.append(torch.zeros(mats[p].nrows, dtype=torch.float64, device="cuda"))
    for p in range(6):
        B.arm(ids[p], bs[p], xs[p], tol=1e-10)
    steps = 0
    while len(done) < len(mats):
        for i, r in B.step(7, mixed=mixed):
            done[i] = r
        steps += 1
        if steps == 3:
            for p in range(6, len(mats)):
                B.arm(ids[p], bs[p], xs[p], tol=1e-10)
        assert steps < 100000
    for p, i in enumerate(ids):
        assert np.array_equal(xs[p].cpu().numpy(), xs_ref[p].cpu().numpy()), p
        assert done[i]["iterations"] == res_ref[p]["iterations"]
        assert done[i]["converged"]
    B.remove(ids[3])
    j = B.add(mats[3])
    assert j == ids[3]
