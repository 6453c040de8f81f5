"""Parity at the benchmark sizes.  The oracle is too slow for many steps at
96^3 (seconds per step), so these compare the first steps directly and use
size-independent properties for the rest: the FP64 GPU step against the
oracle on the full 96^3 cavity (5.3 M tets), the SUPG hexa8 step on a
quarter-size channel, the mixed form against the FP64 GPU form, and bitwise
determinism of repeated full-size runs."""
import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def gpu_run(p, steps, precision=api.FM_FP64):
    g = api.GpuProblem(p, precision)
    b = api.Batch([g])
    b.step(steps)
    b.sync()
    st = g.state()
    b.close()
    g.close()
    return st


def test_vms_96_cubed_two_steps_against_oracle():
    p = mesh.cavity(96, seed=0, steps=200)
    u, pr, _, _ = gpu_run(p, 2)
    o = oracle_b.OracleSolve(p)
    o.step(2)
    st, _, _, _ = o.state()
    eu, ep = rel(u, st[:, :3]), rel(pr, st[:, 3])
    print(f"96^3 VMS after 2 steps: u {eu:.3e} p {ep:.3e}")
    assert eu <= 1e-12 and ep <= 1e-12


def test_vms_96_cubed_deterministic_and_mixed_close():
    p = mesh.cavity(96, seed=1, steps=200)
    a = gpu_run(p, 20)
    b = gpu_run(p, 20)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    m = gpu_run(p, 20, api.FM_MIXED)
    eu, ep = rel(m[0], a[0]), rel(m[1], a[1])
    print(f"96^3 mixed vs FP64 after 20 steps: u {eu:.3e} p {ep:.3e}")
    assert eu <= 1e-6 and ep <= 1e-6


def test_supg_hexa_channel_128x32x32_against_oracle():
    p = mesh.channel(128, 32, 32, seed=0, steps=500)
    u, pr, el, _ = gpu_run(p, 2)
    o = oracle_b.OracleSolve(p)
    o.step(2)
    st, oel, _, _ = o.state()
    eu, ep = rel(u, st[:, :3]), rel(pr, oel[:, 0])
    print(f"SUPG hexa 128x32x32 after 2 steps: u {eu:.3e} element p {ep:.3e}")
    assert eu <= 1e-12 and ep <= 1e-11
