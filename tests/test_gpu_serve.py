"""Served stream (continuous batching): requests that arrive while others are
on the GPU join the running batch; every result must be the same as the same
request solved alone (bitwise: tiles never span problems and every launch is
deterministic), and the FP64 results must match the oracle."""
import numpy as np
import pytest

from femorph_b200 import api, mesh, serve
from oracle import oracle_b

pytestmark = pytest.mark.gpu


def alone(p, steps, precision):
    g = api.GpuProblem(p, precision)
    b = api.Batch([g])
    b.step(steps)
    b.sync()
    u, pr, _, _ = g.state()
    b.close()
    g.close()
    return u, pr


@pytest.mark.parametrize("precision", [api.FM_FP64, api.FM_MIXED])
def test_results_same_alone_and_in_the_mix(precision):
    # arrivals close together (20,000 requests/s), so that several requests
    # are resident at once however fast the host side admits and retires them
    reqs = serve.draw_requests(10, rate=20000.0, seed=3, n_range=(3, 7), steps_range=(5, 40))
    srv = serve.Server(precision=precision, hbm_budget=64 << 20, max_problems=6, block=4, prepare_workers=3)
    stats = srv.run(reqs)
    srv.close()
    assert stats["failed"] == 0 and stats["requests"] == 10
    # several requests were resident at once: their work overlapped on the device
    assert stats["peak_resident"] >= 3
    for r in reqs:
        u0, p0 = alone(r.problem, r.steps, precision)
        u, p = r.result
        assert np.array_equal(u, u0) and np.array_equal(p, p0), r.rid
    if precision == api.FM_FP64:
        r = reqs[0]
        o = oracle_b.OracleSolve(r.problem)
        o.step(r.steps)
        st, _, _, _ = o.state()
        u, p = r.result
        assert np.linalg.norm(u - st[:, :3]) <= 1e-10 * np.linalg.norm(st[:, :3])
        assert np.linalg.norm(p - st[:, 3]) <= 1e-10 * np.linalg.norm(st[:, 3])


def test_budget_admission_waits_for_room():
    # a budget that holds only a couple of these problems at a time: later
    # requests wait until earlier ones retire, and all finish
    reqs = serve.draw_requests(6, rate=1000.0, seed=5, n_range=(6, 6), steps_range=(8, 8))
    per = api.capacity_bytes(mesh.VMS, 4, 4, 3000, 600, api.FM_FP64)
    srv = serve.Server(precision=api.FM_FP64, hbm_budget=per, max_problems=4, block=4, prepare_workers=2)
    stats = srv.run(reqs)
    srv.close()
    assert stats["failed"] == 0
    assert stats["peak_resident"] <= 2
    admitted = sorted(r.admitted for r in reqs)
    done = sorted(r.done for r in reqs)
    assert admitted[-1] >= done[0]   # the last admission had to wait for a retirement


@pytest.mark.parametrize("precision", [api.FM_FP64, api.FM_MIXED])
def test_preempted_solves_resume_bit_for_bit(tmp_path, precision):
    # room for about two of these problems; with preempt_after = 0 a waiting
    # request evicts the resident solve with the most work left after every
    # round, so solves are checkpointed, removed, restored and resumed many
    # times; each result must still equal the request solved alone
    reqs = serve.draw_requests(5, rate=1000.0, seed=9, n_range=(6, 6), steps_range=(24, 40))
    per = api.capacity_bytes(mesh.VMS, 4, 4, 3000, 600, precision)
    srv = serve.Server(precision=precision, hbm_budget=per, max_problems=4, block=4, prepare_workers=2,
                       preempt_after=0.0, spill_dir=str(tmp_path))
    stats = srv.run(reqs)
    srv.close()
    assert stats["failed"] == 0
    assert stats["preemptions"] >= 2 and stats["peak_resident"] <= 2
    assert sum(r.preemptions for r in reqs) == stats["preemptions"]
    assert not list(tmp_path.iterdir())   # every spilled checkpoint was restored and removed
    for r in reqs:
        assert r.steps_done == r.steps
        u0, p0 = alone(r.problem, r.steps, precision)
        u, p = r.result
        assert np.array_equal(u, u0) and np.array_equal(p, p0), r.rid
