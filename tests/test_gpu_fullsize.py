"""Parity at the benchmark sizes and step counts, against the oracle (the
plain-C restatement, pinned bit for bit to the compiled reference, running
its element loops on all host threads).

* 96^3 VMS cavity (5.3 M tets), 200 steps: FP64 within 1e-10 relative L2 of
  the oracle (velocity and pressure) at every 20th step, the mixed form
  within 1e-6 (velocity).  Reference loop: femVMSExplicitFluidSolver.cpp:
  1025-1234.
* SUPG variant of the same cavity (CFL 0.05), 20 steps: FP64 within 1e-10
  (velocity and element pressure), mixed within 1e-6 (velocity).
  Reference loop: femSUPGExplicitFluidSolver.cpp:1034-1643.
* The full 256x64x64 hexa8 channel (1 M hexa), 20 steps against the oracle,
  FP64 and mixed; then 500 steps of the mixed form against the FP64 form.
* The batched workload (256 cavities, n ~ U{8..48}), 200 steps: mixed
  against FP64 per problem.
* Bitwise determinism of repeated full-size runs.

Figures are printed (run pytest with -s to see them)."""
import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED_U = 1e-6


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


class Solve:
    """One GPU solve in its own batch."""

    def __init__(self, p, precision):
        self.g = api.GpuProblem(p, precision)
        self.b = api.Batch([self.g])

    def step(self, n):
        self.b.step(n)

    def state(self):
        self.b.sync()
        return self.g.state()

    def close(self):
        self.b.close()
        self.g.close()


def gpu_run(p, steps, precision=api.FM_FP64):
    s = Solve(p, precision)
    s.step(steps)
    st = s.state()
    s.close()
    return st


def test_vms_96_cubed_200_steps_against_oracle():
    """Config 2 (plain FP64 and mixed) over its 200 steps, checked every 20."""
    p = mesh.cavity(96, seed=0, steps=200)
    f, m = Solve(p, api.FM_FP64), Solve(p, api.FM_MIXED)
    o = oracle_b.OracleSolve(p)
    for s in range(20, 201, 20):
        f.step(20)        # the GPU steps run while the oracle computes
        m.step(20)
        o.step(20)
        st = o.state()[0]
        uf, pf = f.state()[:2]
        um, pm = m.state()[:2]
        eu, ep = rel(uf, st[:, :3]), rel(pf, st[:, 3])
        mu, mp = rel(um, st[:, :3]), rel(pm, st[:, 3])
        print(f"[parity] vms96 step {s}: fp64 u {eu:.3e} p {ep:.3e} | mixed u {mu:.3e} p {mp:.3e}")
        assert eu <= TOL_FP64 and ep <= TOL_FP64, (s, eu, ep)
        assert mu <= TOL_MIXED_U, (s, mu)
        assert mp <= 1e-5, (s, mp)
    f.close()
    m.close()
    o.close()


def test_supg_tet_96_cubed_20_steps_against_oracle():
    """SUPG variant of config 2 (EXOPTS 1 0 1 1 1 1, CFL 0.05)."""
    p = mesh.cavity(96, seed=0, steps=200, solver=mesh.SUPG, cfl=0.05)
    f, m = Solve(p, api.FM_FP64), Solve(p, api.FM_MIXED)
    o = oracle_b.OracleSolve(p)
    for s in (10, 20):
        f.step(10)
        m.step(10)
        o.step(10)
        st, oel, _, _ = o.state()
        uf, pf = f.state()[:2]
        um, pm = m.state()[:2]
        eu, ep = rel(uf, st[:, :3]), rel(pf, oel[:, 0])
        mu, mp = rel(um, st[:, :3]), rel(pm, oel[:, 0])
        print(f"[parity] supg_tet96 step {s}: fp64 u {eu:.3e} element p {ep:.3e} | mixed u {mu:.3e} p {mp:.3e}")
        assert eu <= TOL_FP64 and ep <= TOL_FP64, (s, eu, ep)
        assert mu <= TOL_MIXED_U, (s, mu)
    f.close()
    m.close()
    o.close()


def test_supg_hexa_channel_full_size():
    """Config 3: the full 256x64x64 channel, 20 steps against the oracle in
    FP64 and mixed, then 500 steps of the mixed form against the FP64 form."""
    p = mesh.channel(256, 64, 64, seed=0, steps=500)
    f, m = Solve(p, api.FM_FP64), Solve(p, api.FM_MIXED)
    o = oracle_b.OracleSolve(p)
    for s in (10, 20):
        f.step(10)
        m.step(10)
        o.step(10)
        st, oel, _, _ = o.state()
        uf, pf = f.state()[:2]
        um, pm = m.state()[:2]
        eu, ep = rel(uf, st[:, :3]), rel(pf, oel[:, 0])
        mu, mp = rel(um, st[:, :3]), rel(pm, oel[:, 0])
        print(f"[parity] channel256 step {s}: fp64 u {eu:.3e} element p {ep:.3e} | mixed u {mu:.3e} p {mp:.3e}")
        assert eu <= TOL_FP64 and ep <= TOL_FP64, (s, eu, ep)
        assert mu <= TOL_MIXED_U, (s, mu)
    o.close()
    f.step(480)
    m.step(480)
    uf, pf = f.state()[:2]
    um, pm = m.state()[:2]
    mu, mp = rel(um, uf), rel(pm, pf)
    print(f"[parity] channel256 step 500: mixed vs fp64 u {mu:.3e} element p {mp:.3e}")
    assert mu <= TOL_MIXED_U, mu
    f.close()
    m.close()


def test_batched_cavities_200_steps_mixed_against_fp64():
    """Config 4: the 256 batched cavities in one batch per form, 200 steps;
    the mixed form against the FP64 form, problem by problem."""
    probs = mesh.batched_cavities(256, seed=0, steps=200)
    states = {}
    for name, prec in (("fp64", api.FM_FP64), ("mixed", api.FM_MIXED)):
        gs = [api.GpuProblem(p, prec) for p in probs]
        b = api.Batch(gs, graph_steps=50)
        b.step(200)
        b.sync()
        states[name] = [g.state(elements=False)[:2] for g in gs]
        b.close()
        for g in gs:
            g.close()
    eu = [rel(a[0], b_[0]) for a, b_ in zip(states["mixed"], states["fp64"])]
    ep = [rel(a[1], b_[1]) for a, b_ in zip(states["mixed"], states["fp64"])]
    k = int(np.argmax(eu))
    print(f"[parity] batched256 step 200: mixed vs fp64 u max {max(eu):.3e} (problem {k}, n^3 x 6 = "
          f"{probs[k].n_elems} tets) median {np.median(eu):.3e}; p max {max(ep):.3e} median {np.median(ep):.3e}")
    assert max(eu) <= TOL_MIXED_U, (k, max(eu))


def test_vms_96_cubed_deterministic():
    p = mesh.cavity(96, seed=1, steps=200)
    a = gpu_run(p, 20)
    b = gpu_run(p, 20)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
