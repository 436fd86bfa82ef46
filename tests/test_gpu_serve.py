"""Serving (femd_b200.serve): the heat loop of the reference's example13 served through the
batched solver, results the same alone and in a mix, admission by free device memory."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL = [8, 10, 12, 16, 20]


@pytest.fixture(scope="module")
def sv():
    from femd_b200 import serve
    return serve


@pytest.fixture(scope="module")
def lib(sv):
    return sv.SpaceLibrary()


def example13_session(sv, lib):
    """P2 on rectangle_mesh(0,0,1,1,20,20), dt = 1e-3, w = L2 projection of
    u0 = sin(pi x) sin(pi y) + sin(3 pi x) sin(2 pi y) (example13)."""
    import femd_b200 as fb
    s = lib.get(20, 2)
    Q = s["V"].cache(6)
    F = fb.assemble_vector_2d(Q, [0], [fb.Coef.sinsin(0.0, 1.0, math.pi, math.pi)])
    F += fb.assemble_vector_2d(Q, [0], [fb.Coef.sinsin(0.0, 1.0, 3 * math.pi, 2 * math.pi)])
    M = sv.mass(lib, 20, 2)
    w, conv, its, res, brk = fb.cg_solve(M, fb.JacobiPreconditioner(M), F, None, 10000, 1e-14)
    assert conv
    return sv.HeatSession(lib, 20, 2, 1e-3, u0=w)


def exact13(t):
    return lambda x, y: (np.exp(-2 * np.pi ** 2 * t) * np.sin(np.pi * x) * np.sin(np.pi * y)
                         + np.exp(-13 * np.pi ** 2 * t) * np.sin(3 * np.pi * x) * np.sin(2 * np.pi * y))


@pytest.mark.parametrize("path", ["served_mixed", "served_fp64", "served_lockstep", "served_continuous", "plain"])
def test_example13_heat_loop_pin(sv, lib, path):
    """100 backward-Euler steps to t = 0.1: the reference prints L2 error 1.35e-03."""
    from femd_b200.workloads import l2_error
    S = example13_session(sv, lib)
    trace = [sv.Request(i, 0.0, "heat", session=0) for i in range(100)]
    if path == "plain":
        st = sv.run_plain(lib, [S], trace, tol=1e-12, realtime=False)
    else:
        srv = sv.Server(lib, [S], mixed=(path != "served_fp64"), iters=16, tol=1e-12,
                        engine={"served_lockstep": "lockstep", "served_continuous": "continuous"}.get(path, "persistent"))
        st = srv.run(trace, realtime=False)
    assert st["completed"] == 100 and st["all_converged"]
    err = l2_error(lib.get(20, 2)["V"], S.u, exact13(0.1))
    assert f"{err:.2e}" == "1.35e-03", err


@pytest.mark.parametrize("engine", ["persistent", "lockstep", "continuous"])
def test_served_results_alone_and_in_the_mix(sv, lib, engine):
    sessions = sv.make_sessions(lib, 5, 3, sizes=SMALL)
    trace = sv.make_trace(11, 1e6, 24, len(sessions), sizes=SMALL)
    srv = sv.Server(lib, sessions, mixed=True, iters=8, keep_solutions=True, engine=engine)
    st = srv.run(trace, realtime=False)
    assert st["completed"] == len(trace) and st["all_converged"]
    first_heat = {}
    for r in trace:
        if r.kind == "heat" and r.session not in first_heat:
            first_heat[r.session] = r
    for S in sessions:
        S.reset()
    for r in [r for r in trace if r.kind == "poisson"][:6] + list(first_heat.values()):
        alone = sv.Request(0, 0.0, r.kind, session=r.session, N=r.N, k=r.k, c=r.c, seed=r.seed)
        srv1 = sv.Server(lib, sessions, mixed=True, iters=8, keep_solutions=True, engine=engine)
        srv1.run([alone], realtime=False)
        assert np.array_equal(alone.x.cpu().numpy(), r.x.cpu().numpy()), r
        if r.kind == "heat":
            sessions[r.session].reset()


@pytest.mark.parametrize("engine", ["persistent", "lockstep", "continuous"])
def test_served_matches_plain_fp64(sv, lib, engine):
    sessions = sv.make_sessions(lib, 6, 2, sizes=SMALL)
    trace = sv.make_trace(12, 1e6, 16, len(sessions), sizes=SMALL)
    for S in sessions:
        S.reset()
    srv = sv.Server(lib, sessions, mixed=True, iters=16, keep_solutions=True, tol=1e-12, engine=engine)
    srv.run(trace, realtime=False)
    served = {r.rid: r.x.clone() for r in trace}
    for S in sessions:
        S.reset()
    trace2 = sv.make_trace(12, 1e6, 16, len(sessions), sizes=SMALL)
    sv.run_plain(lib, sessions, trace2, tol=1e-12, realtime=False, keep_solutions=True)
    for r in trace2:
        a, b = served[r.rid].cpu().numpy(), r.x.cpu().numpy()
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b), r


def test_admission_by_free_memory(sv, lib):
    """A fake device free-memory figure and a pool budget that fit one Poisson request at a time:
    requests wait in the queue instead of failing, and all complete."""
    trace = sv.make_trace(13, 1e6, 10, 0, sizes=[16], degrees=(2,))     # equal sizes
    one = max(sv.request_bytes(lib, r, []) for r in trace)
    reserve = 1 << 20
    srv = sv.Server(lib, [], mixed=True, iters=8, reserve_bytes=reserve, free_memory=lambda: reserve + one,
                    hbm_budget=one)
    peak = [0]
    step = srv.batch.step

    def counting_step(iters, mixed=True, **kw):
        peak[0] = max(peak[0], len(srv.active))
        return step(iters, mixed=mixed, **kw)

    srv.batch.step = counting_step
    st = srv.run(trace, realtime=False)
    assert st["completed"] == len(trace) and st["all_converged"]
    assert peak[0] == 1


def test_no_admission_below_the_reserve(sv, lib):
    """With the fake free memory under the reserve nothing is admitted: run() returns when its
    time runs out with every request still queued, and no launch was made."""
    trace = sv.make_trace(14, 1e6, 3, 0, sizes=SMALL)
    srv = sv.Server(lib, [], mixed=True, iters=8, reserve_bytes=1 << 30, free_memory=lambda: 1 << 20)
    st = srv.run(trace, realtime=False, max_seconds=0.5)
    assert st["completed"] == 0 and srv.launches == 0


def test_continuous_admits_mid_flight(sv, lib):
    """Continuous batching: a small request armed while a large one is in flight joins at the next
    chunk boundary, finishes first, and has the same bits as when it is solved alone; the large
    one too."""
    import torch
    from femd_b200.batch import Batch
    big = sv.stiffness(lib, 64, 3, 1.3)
    small = sv.stiffness(lib, 16, 1, 0.7)
    bb = torch.as_tensor(np.random.default_rng(1).standard_normal(big.nrows)).cuda()
    bs = torch.as_tensor(np.random.default_rng(2).standard_normal(small.nrows)).cuda()
    B = Batch()
    ib, is_ = B.add(big), B.add(small)
    xb = torch.zeros(big.nrows, dtype=torch.float64, device="cuda")
    xs = torch.zeros(small.nrows, dtype=torch.float64, device="cuda")
    B.arm(ib, bb, xb)
    fin = B.step(16, mixed=True, engine="continuous")          # the big one alone, 16 iterations
    assert fin == []
    B.arm(is_, bs, xs)                                          # arrives mid-flight
    order = []
    while len(order) < 2:
        order += [i for i, r in B.step(16, mixed=True, engine="continuous")]
    assert order == [is_, ib]
    for K, b, x in ((small, bs, xs), (big, bb, xb)):
        xa, ra = Batch([K]).solve([b], mixed=True, engine="lockstep")
        assert ra[0]["converged"]
        assert np.array_equal(xa[0].cpu().numpy(), x.cpu().numpy())


def test_large_requests_on_the_whole_gpu_path(sv, lib):
    """big_nnz: requests whose matrix reaches it are solved one at a time by the fused FP64 CG
    between batch steps -- the plain path's solve, so their solutions are the plain path's bits;
    the batched ones stay within 1e-8 of plain FP64."""
    sizes = [8, 12, 20, 24]
    big = lib.get(20, 2)["nnz"]                       # every (20, 2) or larger request goes direct
    sessions = sv.make_sessions(lib, 7, 2, sizes=sizes)
    trace = sv.make_trace(13, 1e6, 16, len(sessions), sizes=sizes)
    for S in sessions:
        S.reset()
    srv = sv.Server(lib, sessions, mixed=True, iters=16, keep_solutions=True, tol=1e-12, engine="continuous", big_nnz=big)
    st = srv.run(trace, realtime=False)
    assert st["completed"] == len(trace) and st["all_converged"]
    served = {r.rid: r.x.clone() for r in trace}
    for S in sessions:
        S.reset()
    trace2 = sv.make_trace(13, 1e6, 16, len(sessions), sizes=sizes)
    sv.run_plain(lib, sessions, trace2, tol=1e-12, realtime=False, keep_solutions=True)
    ndirect = 0
    for r in trace2:
        nnz = (sessions[r.session].A.nnz if r.kind == "heat" else lib.get(r.N, r.k)["nnz"])
        a, b = served[r.rid].cpu().numpy(), r.x.cpu().numpy()
        if nnz >= big:                                # a large session's every step is on the direct path
            ndirect += 1
            assert np.array_equal(a, b), r
        else:
            assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b), r
    assert ndirect > 0
