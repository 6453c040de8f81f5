"""fm_vms_solve_static: the VMS solve for callers that cannot call cudaMalloc
(device memory already held by another allocator, or a latency-bound path
on which cudaMalloc/cudaFree's device-wide synchronisation is not
acceptable).  It keeps everything in one fixed device array, so two calls
in a row must not see each other's leftovers.  Each call is checked, through
the C ABI, against the allocating path (fm_batch_create + fm_batch_step +
fm_problem_get_state): the two paths run the same kernels on the same tile
layout in the same order, so their results must be equal bit for bit (any
leftover state of the previous call would break that).  Each call is also
checked against the oracle with the per-step tolerance of the parity tests.

This file sorts last so that a run stopping at the first failure has run
every other test before it."""
import ctypes as C

import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def allocating_path(p, steps):
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.step(steps)
    b.sync()
    u, pr, _, _ = g.state()
    b.close()
    g.close()
    return u, pr


def static_path(p, steps):
    g = api.GpuProblem(p)
    g.prepare()
    u = np.full((p.n_nodes, 3), np.nan)
    pr = np.full(p.n_nodes, np.nan)
    rc = api.lib().fm_vms_solve_static(g.h, steps, 0, u.ctypes.data, pr.ctypes.data, None)
    api.check(rc)
    g.close()
    return u, pr


def test_two_calls_in_a_row_match_allocating_path():
    # different sizes, BC tables and dual iterations, so anything the first
    # call leaves in the array would show up in the second
    p1 = mesh.cavity(6, seed=71, steps=5, lid=0.8)
    p2 = mesh.cavity(4, seed=72, steps=4, lid=1.2)
    p2.tot_dual_steps = 1
    p2.dual_step = 0.5 * p2.time_step
    n = p2.vel_node.size
    p2.vel_node = np.concatenate([p2.vel_node, p2.vel_node]).astype(np.int32)
    ramp = np.zeros((2 * n, 4))
    ramp[n:, 0] = 1.2
    ramp[n:, 3] = 2.0 * p2.time_step
    p2.vel_vals = ramp
    p2.vel_dir = np.full(2 * n, 6, np.int32)
    for p, steps in ((p1, 5), (p2, 4)):
        u, pr = static_path(p, steps)
        u0, pr0 = allocating_path(p, steps)
        assert np.isfinite(u).all() and np.isfinite(pr).all()
        assert np.array_equal(u, u0) and np.array_equal(pr, pr0), (rel(u, u0), rel(pr, pr0))
        o = oracle_b.OracleSolve(p)
        o.step(steps)
        st = o.state()[0]
        o.close()
        assert rel(u, st[:, :3]) <= TOL and rel(pr, st[:, 3]) <= TOL, (rel(u, st[:, :3]), rel(pr, st[:, 3]))


def test_rejects_problems_beyond_the_array():
    p = mesh.cavity(36, seed=73, steps=1)
    g = api.GpuProblem(p)
    g.prepare()
    rc = api.lib().fm_vms_solve_static(g.h, 1, 0, None, None, None)
    assert rc == api.FM_ERR_INVALID
    assert b"limit" in api.lib().fm_last_error_message()
    g.close()
