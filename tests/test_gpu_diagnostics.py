"""VMS diagnostics (the reference's per-dual-iteration log row and its
res_v / res_p fields): one row per dual iteration of every problem that
stepped, in step / dual-iteration order, with the reference's time
accumulation; turning them on changes nothing in the solve; problems that
join a pool later get them too.  Values against the compiled reference:
tests/test_gpu_dropin.py."""
import numpy as np
import pytest

from femorph_b200 import api, mesh

pytestmark = pytest.mark.gpu


def _problem(n=4, seed=51, dual=2):
    p = mesh.cavity(n, seed=seed, steps=10, lid=0.9)
    p.tot_dual_steps = dual
    return p


def test_rows_one_per_dual_iteration_and_state_unchanged():
    p = _problem()
    ref = api.GpuProblem(p)
    b0 = api.Batch([ref])
    b0.step(4)
    b0.sync()
    u0, p0, _, s0 = ref.state()
    b0.close()
    ref.close()
    g = api.GpuProblem(p)
    b = api.Batch([g], graph_steps=2)
    b.set_diagnostics(True)
    b.step(3)
    b.step(1)
    b.sync()
    rows = g.vms_log()
    assert rows.shape == (4 * 3, 6)
    steps, duals = rows[:, 0].astype(int), rows[:, 1].astype(int)
    assert list(steps) == [s for s in range(4) for _ in range(3)]
    assert list(duals) == [1, 2, 3] * 4
    t = 0.0
    for s in range(4):
        t += p.time_step
        assert np.all(rows[steps == s, 2] == t)
    assert np.all(rows[:, 3:] >= 0) and np.all(np.isfinite(rows))
    assert g.vms_log().shape == (0, 6)          # the queue was emptied
    ru, rp = g.vms_residuals()
    assert ru.shape == (p.n_elems, 3) and rp.shape == (p.n_elems,)
    # the row's maxima are those of the last iteration's centroid residuals
    assert np.isclose(np.linalg.norm(ru, axis=1).max(), rows[-1, 3], rtol=1e-14)
    assert np.isclose(np.abs(rp).max(), rows[-1, 4], rtol=1e-14)
    u, pr, _, sd = g.state()
    assert np.array_equal(u, u0) and np.array_equal(pr, p0) and np.array_equal(sd, s0)
    b.set_diagnostics(False)   # graphs are captured again without the residual buffer
    b.step(2)
    b.sync()
    assert g.vms_log().shape == (0, 6)
    b.close()
    g.close()


def test_pool_members_added_later_get_rows():
    pa, pb = _problem(4, 52, 0), _problem(3, 53, 1)
    pool = api.Pool(mesh.VMS, 4, max_problems=3, max_elems=pa.n_elems + pb.n_elems,
                    max_nodes=pa.n_nodes + pb.n_nodes)
    ga = api.GpuProblem(pa)
    assert pool.add(ga)
    api.check(api.lib().fm_batch_set_diagnostics(pool.h, 1))
    gb = api.GpuProblem(pb)
    assert pool.add(gb)
    pool.step([ga, gb], [3, 2])
    pool.sync()
    ra, rb = ga.vms_log(), gb.vms_log()
    assert ra.shape == (3, 6) and rb.shape == (4, 6)
    assert list(rb[:, 0].astype(int)) == [0, 0, 1, 1] and list(rb[:, 1].astype(int)) == [1, 2, 1, 2]
    pool.remove(ga)
    pool.close()


def test_diagnostics_refused_for_supg():
    g = api.GpuProblem(mesh.cavity(3, seed=1, steps=2, solver=mesh.SUPG))
    b = api.Batch([g])
    with pytest.raises(api.FmError) as ei:
        b.set_diagnostics(True)
    assert ei.value.code == api.FM_ERR_INVALID
    b.close()
    g.close()
