"""The Poisson solver (femPoissonSolver::solve, femSolver.cpp:409-654) on the
GPU against the oracle: the reference's own element arithmetic (pinned bit
for bit in tests/test_poisson.py), assembled with its sources, face Neumann
values and Dirichlet rows, solved directly.  The reference itself solves only
through Trilinos, so the bar is the solution of the same system: relative L2
<= 1e-10 at a CG tolerance of 1e-14."""
import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def gpu_solve(p, tol=1e-14, max_iter=20000):
    s = api.GpuPoisson(p)
    it, rr, ms = s.solve(tol, max_iter)
    x, d = s.solution()
    s.close()
    return x, d, it, rr


@pytest.mark.parametrize("elem_type,n", [(mesh.TET4, 8), (mesh.HEXA8, 8)])
def test_classic_against_oracle(elem_type, n):
    """Anisotropic per-element diffusivity, element sources, face Neumann
    values on x = 1, Dirichlet values on x = 0."""
    p = mesh.poisson_box(n, elem_type=elem_type, seed=11)
    x, _, it, rr = gpu_solve(p)
    xo, _ = oracle_b.poisson_solve(p)
    e = rel(x, xo)
    print(f"[parity] poisson {p.name}: {it} CG iterations, rel residual {rr:.2e}, rel L2 {e:.2e}")
    assert rr <= 1e-14 and e <= TOL
    assert np.array_equal(x[p.dir_node], p.dir_value)


def test_ppe_pure_neumann_against_oracle():
    """PPE without Dirichlet rows (singular K): the zero-sum part of the
    right-hand side, the solution's average subtracted."""
    p = mesh.poisson_box(8, problem=mesh.POISSON_PPE, seed=4, dirichlet=False)
    x, _, it, rr = gpu_solve(p)
    xo, _ = oracle_b.poisson_solve(p)
    e = rel(x, xo)
    print(f"[parity] poisson PPE {p.name}: {it} iterations, rel L2 {e:.2e}")
    assert abs(x.mean()) <= 1e-13 * np.abs(x).max()
    assert e <= TOL


@pytest.mark.parametrize("elem_type", [mesh.TET4, mesh.HEXA8])
def test_distance_against_oracle(elem_type):
    p = mesh.poisson_box(6, elem_type=elem_type, problem=mesh.POISSON_DISTANCE, seed=8)
    x, d, it, rr = gpu_solve(p)
    xo, do = oracle_b.poisson_solve(p)
    ok = np.isfinite(do)
    assert np.array_equal(np.isfinite(d), ok)
    assert rel(x, xo) <= TOL and rel(d[ok], do[ok]) <= TOL


def test_deterministic_and_iteration_limit():
    p = mesh.poisson_box(6, seed=3)
    x1, _, it1, _ = gpu_solve(p)
    x2, _, it2, _ = gpu_solve(p)
    assert it1 == it2 and np.array_equal(x1, x2)
    s = api.GpuPoisson(p)
    it, rr, _ = s.solve(1e-14, 7)
    assert it == 7 and rr > 1e-14
    # a second solve on the same system starts again from x = 0
    it_b, _, _ = s.solve(1e-14, 20000)
    x3, _ = s.solution()
    s.close()
    assert it_b == it1 and np.array_equal(x3, x1)


def test_zero_right_hand_side():
    p = mesh.poisson_box(4, sources=False, neumann=False, dirichlet=True)
    p.dir_value = np.zeros_like(p.dir_value)
    x, _, it, rr = gpu_solve(p)
    assert it == 0 and not x.any()


def test_dropin_poisson_adapter(tmp_path):
    """The femSolver adapter (femorph_b200/adapter/femPoissonSolverGPU) behind
    the reference's own .dat reader and FixedElementConnectivities
    (oracle/_ref/fm_gpudrv): its "PoissonResult" and "cellDistance" fields
    against the oracle."""
    import os
    import subprocess

    from oracle import ref
    gpudrv = os.path.join(os.path.dirname(ref.REFDRV), "fm_gpudrv")
    if not os.path.exists(gpudrv):
        pytest.skip("oracle/_ref/fm_gpudrv not built")
    p = mesh.poisson_box(5, problem=mesh.POISSON_DISTANCE, seed=6)
    dat = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, dat)
    r = subprocess.run([gpudrv, dat, "poisson-gpu", "--dump", str(tmp_path)], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = ref.read_dump(str(tmp_path / "poisson.f64"))
    xo, do = oracle_b.poisson_solve(p)
    x = out["PoissonResult"][:, 0]
    d = out["cellDistance"][:, 0]
    ok = np.isfinite(do)
    assert rel(x, xo) <= TOL and rel(d[ok], do[ok]) <= TOL


@pytest.mark.parametrize("elem_type,problem", [(mesh.TET4, mesh.POISSON_CLASSIC), (mesh.HEXA8, mesh.POISSON_DISTANCE)])
def test_read_dat_equals_arrays(tmp_path, elem_type, problem):
    """The .dat path (fm_poisson_read_dat) builds the same system as the
    arrays: bitwise the same solution."""
    p = mesh.poisson_box(5, elem_type=elem_type, problem=problem, seed=9)
    dat = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, dat)
    x, d, it, _ = gpu_solve(p)
    s = api.GpuPoisson.read_dat(dat)
    assert s.model() == (p.n_nodes, p.n_elems, p.conn.shape[1], problem)
    it2, _, _ = s.solve(1e-14, 20000)
    x2, d2 = s.solution()
    s.close()
    assert it2 == it and np.array_equal(x2, x)
    if d is not None:
        assert np.array_equal(d2, d, equal_nan=True)


@pytest.mark.parametrize("problem", [mesh.POISSON_CLASSIC, mesh.POISSON_DISTANCE])
def test_vtk_writer_matches_reference_exporter(tmp_path, problem):
    """fm_poisson_write_vtk against the reference's own exporter
    (femModel::ExportToVTKLegacy) run on the same solution: the adapter
    behind the reference's reader (oracle/_ref/fm_gpudrv poisson-gpu --vtk)
    and the library from the same .dat file at the same tolerance give the
    same bytes."""
    import os
    import subprocess

    from oracle import ref
    gpudrv = os.path.join(os.path.dirname(ref.REFDRV), "fm_gpudrv")
    if not os.path.exists(gpudrv):
        pytest.skip("oracle/_ref/fm_gpudrv not built")
    p = mesh.poisson_box(4, problem=problem, seed=12)
    dat = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, dat)
    r = subprocess.run([gpudrv, dat, "poisson-gpu", "--dump", str(tmp_path), "--vtk"], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    s = api.GpuPoisson.read_dat(dat)
    assert s.model() == (p.n_nodes, p.n_elems, p.conn.shape[1], problem)
    s.solve(1e-14, 100000)
    mine = str(tmp_path / "mine.vtk")
    s.write_vtk(mine)
    s.close()
    assert open(mine).read() == open(str(tmp_path / "poisson")).read()
