"""Continuous batching: problems join and leave a batch with fixed device
pools between launches.  A problem's results must not depend on which other
problems share its batch, on where in the pools it was placed, or on what
was placed there before (bitwise equality with the problem solved alone),
and the stepped state must match the oracle."""
import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def alone(p, steps, precision=api.FM_FP64, **tuning):
    g = api.GpuProblem(p, precision)
    b = api.Batch([g], **tuning)
    b.step(steps)
    b.sync()
    st = g.state()
    b.close()
    g.close()
    return st


def test_join_leave_bitwise_equal_to_alone():
    pa = mesh.cavity(4, seed=21, steps=8, lid=0.7)
    pb = mesh.cavity(5, seed=22, steps=8, lid=1.1)
    pc = mesh.cavity(3, seed=23, steps=8, lid=0.9)
    ref_b = alone(pb, 7)
    ref_c = alone(pc, 5)
    E = pa.n_elems + pb.n_elems + pc.n_elems
    N = pa.n_nodes + pb.n_nodes + pc.n_nodes
    pool = api.Pool(mesh.VMS, 4, max_problems=4, max_elems=E, max_nodes=N)
    ga, gb, gc = api.GpuProblem(pa), api.GpuProblem(pb), api.GpuProblem(pc)
    assert pool.add(ga) and pool.add(gb)
    pool.step([ga, gb], [3, 2])
    pool.remove(ga)            # leaves; its ranges are reused by pc
    assert pool.add(gc)
    pool.step([gb, gc], [5, 5])
    pool.sync()
    u, pr, _, sd = gb.state()
    assert np.array_equal(u, ref_b[0]) and np.array_equal(pr, ref_b[1]) and np.array_equal(sd, ref_b[3])
    u, pr, _, sd = gc.state()
    assert np.array_equal(u, ref_c[0]) and np.array_equal(pr, ref_c[1]) and np.array_equal(sd, ref_c[3])
    o = oracle_b.OracleSolve(pc)
    o.step(5)
    st, _, _, _ = o.state()
    assert rel(u, st[:, :3]) <= 1e-12 and rel(pr, st[:, 3]) <= 1e-12
    r = pool.resident()
    assert r["problems"] == 2 and r["elems"] == pb.n_elems + pc.n_elems
    pool.close()


def test_capacity_exhausted_reports_oom_and_changes_nothing():
    pa = mesh.cavity(4, seed=31, steps=4)
    pb = mesh.cavity(4, seed=32, steps=4)
    ref = alone(pa, 4)
    pool = api.Pool(mesh.VMS, 4, max_problems=2, max_elems=pa.n_elems + 64, max_nodes=pa.n_nodes + 16)
    ga, gb = api.GpuProblem(pa), api.GpuProblem(pb)
    assert pool.add(ga)
    assert not pool.add(gb)   # no room: FM_ERR_OOM, ga untouched
    pool.step([ga], [4])
    pool.sync()
    u, pr, _, _ = ga.state()
    assert np.array_equal(u, ref[0]) and np.array_equal(pr, ref[1])
    pool.close()


def test_idle_problems_do_not_move_and_graph_replay():
    ps = [mesh.cavity(3, seed=40 + i, steps=12) for i in range(3)]
    refs = [alone(p, 12) for p in ps]
    start1 = alone(ps[1], 0)
    pool = api.Pool(mesh.VMS, 4, max_problems=3, max_elems=sum(p.n_elems for p in ps),
                    max_nodes=sum(p.n_nodes for p in ps), graph_steps=4)
    gs = [api.GpuProblem(p) for p in ps]
    for g in gs:
        assert pool.add(g)
    pool.step(gs[:1], [12])        # graph blocks for the first, others idle
    pool.sync()
    u1, p1, _, _ = gs[1].state()
    assert np.array_equal(u1, start1[0]) and np.array_equal(p1, start1[1])
    pool.step(gs[1:], [12, 12])
    pool.sync()
    for g, r in zip(gs, refs):
        u, pr, _, _ = g.state()
        assert np.array_equal(u, r[0]) and np.array_equal(pr, r[1])
    pool.close()


def test_mixed_precision_pool_matches_alone():
    p1 = mesh.cavity(4, seed=51, steps=6)
    p2 = mesh.cavity(5, seed=52, steps=6)
    r1 = alone(p1, 6, api.FM_MIXED)
    r2 = alone(p2, 6, api.FM_MIXED)
    pool = api.Pool(mesh.VMS, 4, max_problems=2, max_elems=p1.n_elems + p2.n_elems,
                    max_nodes=p1.n_nodes + p2.n_nodes, precision=api.FM_MIXED)
    g1, g2 = api.GpuProblem(p1, api.FM_MIXED), api.GpuProblem(p2, api.FM_MIXED)
    assert pool.add(g2) and pool.add(g1)
    pool.step([g1, g2], [6, 6])
    pool.sync()
    for g, r in ((g1, r1), (g2, r2)):
        u, pr, _, sd = g.state()
        assert np.array_equal(u, r[0]) and np.array_equal(pr, r[1]) and np.array_equal(sd, r[3])
    pool.close()


def test_supg_pool_matches_alone():
    p1 = mesh.channel(8, 4, 4, seed=61, steps=5)
    p2 = mesh.channel(6, 4, 3, seed=62, steps=5, ex_opts=(0, 1, 1, 1, 1, 1))
    r1 = alone(p1, 5)
    r2 = alone(p2, 5)
    pool = api.Pool(mesh.SUPG, 8, max_problems=3, max_elems=2 * (p1.n_elems + p2.n_elems),
                    max_nodes=2 * (p1.n_nodes + p2.n_nodes))
    g1, g2 = api.GpuProblem(p1), api.GpuProblem(p2)
    assert pool.add(g1) and pool.add(g2)
    pool.step([g1, g2], [5, 5])
    pool.sync()
    for g, r in ((g1, r1), (g2, r2)):
        u, pr, el, _ = g.state()
        assert np.array_equal(u, r[0]) and np.array_equal(pr, r[1]) and np.array_equal(el, r[2])
    pool.close()
