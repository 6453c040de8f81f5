"""Checkpoint and restart.  A solve checkpointed after k steps and restored
into a fresh problem object in a fresh batch (or in a pool beside another
problem) must continue exactly: after k more steps its state equals the
uninterrupted 2k-step solve bit for bit, for both solvers and precisions.
Files of another mesh or configuration are refused, and a truncated file
leaves the problem's state untouched."""
import ctypes as C
import os

import numpy as np
import pytest

from femorph_b200 import api, mesh

pytestmark = pytest.mark.gpu


def steps_done(g):
    s = C.c_int64()
    api.check(api.lib().fm_problem_info(g.h, None, None, None, None, C.byref(s)))
    return s.value


def vms_problem(n=5, seed=31):
    p = mesh.cavity(n, seed=seed, steps=20, lid=0.9)
    p.tot_dual_steps = 2  # three dual iterations a step: the pending state spans them
    return p


def supg_problem(hexa=False):
    if hexa:
        return mesh.channel(6, 3, 3, seed=4, steps=20, ex_opts=(0, 0, 1, 1, 1, 1), noise=1e-3)
    p = mesh.cavity(5, seed=32, steps=20, solver=mesh.SUPG)
    p.ex_opts = (0, 0, 1, 1, 1, 1)  # AB2: the element history is part of the state
    return p


def uninterrupted(p, precision, steps):
    g = api.GpuProblem(p, precision)
    b = api.Batch([g])
    b.step(steps)
    b.sync()
    st = g.state()
    b.close()
    g.close()
    return st


def same_state(a, b):
    for x, y in zip(a, b):
        if x is None:
            assert y is None
        else:
            assert np.array_equal(x, y)


CASES = [
    ("vms_fp64", vms_problem, api.FM_FP64),
    ("vms_mixed", vms_problem, api.FM_MIXED),
    ("supg_tet_ab2", supg_problem, api.FM_FP64),
    ("supg_hexa_ab2_mixed", lambda: supg_problem(hexa=True), api.FM_MIXED),
]


@pytest.mark.parametrize("name,make,precision", CASES, ids=[c[0] for c in CASES])
def test_restart_continues_bit_for_bit(tmp_path, name, make, precision):
    k = 4
    ref = uninterrupted(make(), precision, 2 * k)
    path = str(tmp_path / f"{name}.fmck")
    g = api.GpuProblem(make(), precision)
    b = api.Batch([g])
    b.step(k)
    b.sync()
    g.checkpoint(path)
    half = g.state()
    b.close()
    g.close()
    assert os.path.getsize(path) > 160
    # a fresh problem object in a fresh batch
    g2 = api.GpuProblem(make(), precision)
    b2 = api.Batch([g2])
    g2.restore(path)
    assert steps_done(g2) == k
    same_state(g2.state(), half)
    b2.step(k)
    b2.sync()
    assert steps_done(g2) == 2 * k
    same_state(g2.state(), ref)
    b2.close()
    g2.close()


def test_restore_into_pool_beside_another_problem(tmp_path):
    k = 3
    p = vms_problem()
    other = mesh.cavity(4, seed=33, steps=20, lid=1.2)
    ref = uninterrupted(vms_problem(), api.FM_FP64, 2 * k)
    ref_other = uninterrupted(other, api.FM_FP64, k)
    path = str(tmp_path / "pool.fmck")
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.step(k)
    b.sync()
    g.checkpoint(path)
    b.close()
    g.close()
    pool = api.Pool(mesh.VMS, 4, max_problems=3, max_elems=p.n_elems + other.n_elems,
                    max_nodes=p.n_nodes + other.n_nodes)
    go, gr = api.GpuProblem(other), api.GpuProblem(vms_problem())
    assert pool.add(go) and pool.add(gr)
    gr.restore(path)
    pool.step([go, gr], [k, k])
    pool.sync()
    same_state(gr.state(), ref)
    same_state(go.state(), ref_other)
    pool.close()


def test_foreign_and_truncated_files_refused(tmp_path):
    path = str(tmp_path / "a.fmck")
    g = api.GpuProblem(vms_problem())
    b = api.Batch([g])
    b.step(2)
    b.sync()
    g.checkpoint(path)
    before = g.state()
    # another mesh
    h = api.GpuProblem(vms_problem(n=4))
    bh = api.Batch([h])
    with pytest.raises(api.FmError) as ei:
        h.restore(path)
    assert ei.value.code == api.FM_ERR_INVALID
    bh.close()
    h.close()
    # the same mesh with another time step, and with another lid speed
    for change in ("dt", "lid"):
        q = vms_problem()
        if change == "dt":
            q.time_step *= 1.5
        else:
            q.vel_vals = np.array(q.vel_vals) * 1.1
        h = api.GpuProblem(q)
        bh = api.Batch([h])
        with pytest.raises(api.FmError) as ei:
            h.restore(path)
        assert ei.value.code == api.FM_ERR_INVALID, change
        bh.close()
        h.close()
    assert not os.path.exists(path + ".tmp")
    # the same mesh in the other precision
    m = api.GpuProblem(vms_problem(), api.FM_MIXED)
    bm = api.Batch([m])
    with pytest.raises(api.FmError) as ei:
        m.restore(path)
    assert ei.value.code == api.FM_ERR_INVALID
    bm.close()
    m.close()
    # a truncated file: refused before the device state is touched
    data = open(path, "rb").read()
    cut = str(tmp_path / "cut.fmck")
    with open(cut, "wb") as f:
        f.write(data[: len(data) // 2])
    with pytest.raises(api.FmError) as ei:
        g.restore(cut)
    assert ei.value.code == api.FM_ERR_IO
    same_state(g.state(), before)
    with pytest.raises(api.FmError) as ei:
        g.restore(str(tmp_path / "missing.fmck"))
    assert ei.value.code == api.FM_ERR_IO
    b.close()
    g.close()


def test_partition_parts_restart_bit_for_bit(tmp_path):
    """Every part of a mesh split over a batch checkpointed after k steps and
    restored into fresh parts continues exactly (the exchange carries no
    state from one iteration to the next)."""
    k, n = 3, 3
    p = vms_problem(n=6, seed=34)

    def parts_state(full, steps, restore_from=None, save_to=None):
        parts = [full.part(n, q) for q in range(n)]
        b = api.Batch(parts)
        if restore_from:
            for q, part in enumerate(parts):
                part.restore(restore_from[q])
        b.step(steps)
        b.sync()
        if save_to:
            for q, part in enumerate(parts):
                part.checkpoint(save_to[q])
        st = [part.state() for part in parts]
        b.close()
        for part in parts:
            part.close()
        return st

    full = api.GpuProblem(p)
    ref = parts_state(full, 2 * k)
    paths = [str(tmp_path / f"part{q}.fmck") for q in range(n)]
    parts_state(full, k, save_to=paths)
    again = parts_state(full, k, restore_from=paths)
    full.close()
    for a, b in zip(again, ref):
        same_state(a, b)
