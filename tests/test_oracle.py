"""Pins the oracles: oracle B (plain-C restatement) against oracle A (the
compiled reference) and against the reference's own known-answer vector."""
import os
import subprocess

import numpy as np
import pytest

from femorph_b200 import mesh
from oracle import oracle_b, ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _need_oracle_a():
    # oracle/build_ref.sh compiles the reference where its sources are
    # (FEMORPH_REFERENCE); status 2 = sources absent -> skip
    if not ref.available():
        rc = subprocess.call([os.path.join(ROOT, "oracle", "build_ref.sh")], stderr=subprocess.DEVNULL)
        assert rc in (0, 2), rc
    if not ref.available():
        pytest.skip("oracle A (compiled reference) not available")


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _compare_vms(p, steps):
    A = ref.run(p)
    B = oracle_b.OracleSolve(p)
    st, _, _, _ = B.state()
    assert np.array_equal(st[:, :3], A[0]["velocity"])
    checked = 0
    for s in range(1, steps + 1):
        B.step(1)
        st, el, _, t = B.state()
        if s in A:
            d = A[s]
            assert np.array_equal(st[:, :3], d["velocity"]), s
            assert np.array_equal(st[:, 3:], d["pressure"]), s
            assert np.array_equal(el, d["subgrid_u"]), s
            assert t == d["time"]
            checked += 1
    assert checked >= steps - 2


def test_oracle_b_bitexact_vms_cavity():
    _need_oracle_a()
    p = mesh.cavity(4, seed=11, steps=6)
    p.save_every = 1
    _compare_vms(p, 6)


def test_oracle_b_bitexact_vms_dual_steps_and_tables():
    """Dual iterations > 0, a piecewise-linear lid table and the velNodesDir
    row/node quirk (src/femModel.cpp:4549-4576) all reproduced."""
    _need_oracle_a()
    p = mesh.cavity(3, seed=5, steps=5)
    p.save_every = 1
    p.tot_dual_steps = 2
    p.dual_step = p.time_step * 0.5
    # two-row time tables on the lid (ramp), dirs vary per row
    n = p.vel_node.size
    rows_node = np.concatenate([p.vel_node, p.vel_node])
    v0 = np.zeros((n, 4)); v0[:, 3] = 0.0
    v1 = np.zeros((n, 4)); v1[:, 0] = 1.0; v1[:, 1] = 0.3; v1[:, 3] = 3 * p.time_step
    order = np.argsort(-rows_node, kind="stable")  # unsorted file order
    p.vel_node = rows_node[order].astype(np.int32)
    p.vel_vals = np.concatenate([v0, v1])[order]
    p.vel_dir = np.where(np.arange(2 * n) % 3 == 0, 6, 3).astype(np.int32)
    _compare_vms(p, 5)


def test_oracle_b_bitexact_supg_hexa():
    _need_oracle_a()
    p = mesh.channel(6, 3, 3, seed=2, steps=5)
    p.save_every = 1
    A = ref.run(p)
    B = oracle_b.OracleSolve(p)
    for s in range(1, 6):
        B.step(1)
        st, el, _, _ = B.state()
        if s in A:
            d = A[s]
            assert np.array_equal(st[:, :3], d["velocity"])
            assert np.array_equal(el[:, 0:1], d["pressure"])
            assert np.array_equal(el[:, 1:2], d["lambda"])
            assert np.array_equal(el[:, 2:3], d["regime"])


def test_oracle_b_bitexact_supg_hexa_ab2_bbar():
    _need_oracle_a()
    p = mesh.channel(5, 3, 2, seed=4, steps=4, ex_opts=(0, 1, 1, 1, 1, 1))
    p.save_every = 1
    p.glob_fixed = "Z"
    A = ref.run(p)
    B = oracle_b.OracleSolve(p)
    for s in range(1, 5):
        B.step(1)
        st, el, _, _ = B.state()
        if s in A:
            assert np.array_equal(st[:, :3], A[s]["velocity"])
            assert np.array_equal(el[:, 0:1], A[s]["pressure"])


def test_oracle_b_bitexact_supg_tet():
    _need_oracle_a()
    p = mesh.cavity(3, seed=3, steps=4, solver=mesh.SUPG)
    p.save_every = 1
    A = ref.run(p)
    B = oracle_b.OracleSolve(p)
    for s in range(1, 5):
        B.step(1)
        st, el, _, _ = B.state()
        if s in A:
            assert np.array_equal(st[:, :3], A[s]["velocity"])
            assert np.array_equal(el[:, 0:1], A[s]["pressure"])


def test_lumped_mass_known_answer():
    """Reference KAT: example 06 lumped_mass.txt (rho = 10) on its own mesh,
    reproduced to the precision of the 9-digit coordinates it was built from."""
    k = np.load(os.path.join(ROOT, "tests", "golden", "lumped_mass_kat.npz"))
    p = mesh.Problem(coords=k["coords"], conn=k["conn"], solver=mesh.SUPG,
                     props=(float(k["rho"]), 0.01, 0.05, 4.0, 0.0), max_node_dofs=3)
    _, _, lm, _ = oracle_b.OracleSolve(p).state()
    got = lm[k["check_nodes"]]
    want = k["lumped_mass"]
    assert np.max(np.abs(got - want) / np.abs(want)) < 2e-7
    # sum of the complete rows = rho * volume of their support, all positive
    assert np.all(got > 0)


@pytest.mark.parametrize("kind", ["vms_dual", "supg_hexa_ab2", "supg_tet"])
def test_oracle_b_thread_count_independent(kind):
    """The element loops run on host threads and the nodal sums per node in
    element order: one thread and several give identical bits."""
    if kind == "vms_dual":
        p = mesh.cavity(9, seed=3, steps=4)
        p.tot_dual_steps = 1
    elif kind == "supg_hexa_ab2":
        p = mesh.channel(16, 6, 6, seed=2, steps=4, ex_opts=(0, 1, 1, 1, 1, 1))
    else:
        p = mesh.cavity(8, seed=4, steps=4, solver=mesh.SUPG, cfl=0.05)
    out = []
    old = oracle_b.get_threads()
    try:
        for t in (1, 7):
            oracle_b.set_threads(t)
            o = oracle_b.OracleSolve(p)
            o.step(4)
            out.append(o.state())
            o.close()
    finally:
        oracle_b.set_threads(old)
    for a, b in zip(out[0][:3], out[1][:3]):
        assert np.array_equal(a, b)
