"""The replicas path (femd_b200.replicas) as world-size-2 gloo processes on the CPU: the max over
ranks, the whole-job value, and a rank that never reaches the collective, which ends the other
rank's collective with an error after the short process-group timeout instead of a hang."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, out):
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import importlib.util
    spec = importlib.util.spec_from_file_location("replicas", os.path.join(ROOT, "femd_b200", "replicas.py"))
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    dist = R.init("gloo", timeout_s=5.0)
    try:
        if mode == "ok":
            t = 1.0 + rank                                   # rank 1 is the slowest
            tmax = R.max_over_ranks(t, dist, "cpu")
            out.put((rank, tmax, R.whole_job_value(256, world, tmax)))
            R.finish(dist)
        else:
            if rank == 1:
                out.put((rank, "left", None))                # leaves between steps, no collective in flight
                return
            try:
                R.max_over_ranks(1.0, dist, "cpu")
                out.put((rank, "no error", None))
            except Exception as e:                           # the short timeout ends the collective
                out.put((rank, "error", type(e).__name__))
    finally:
        pass


@pytest.mark.parametrize("mode", ["ok", "missing"])
def test_two_gloo_ranks(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=90)
    alive = [p for p in ps if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive
    res = sorted(q.get(timeout=5) for _ in range(2))
    if mode == "ok":
        assert [r[1] for r in res] == [2.0, 2.0]             # every rank sees the slowest time
        assert res[0][2] == pytest.approx(2 * 256 / 2.0)     # whole job / slowest rank
    else:
        assert res[0][1] == "error" and res[1][1] == "left"
