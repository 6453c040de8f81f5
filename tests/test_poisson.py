"""CPU checks of the Poisson path (femPoissonSolver::solve,
femSolver.cpp:409-654): the oracle's element arithmetic against the
reference's own (oracle A, the compiled reference sources), the oracle's
direct solution against the equations it solves, and the C ABI's input
checks (no GPU needed: the host assembly runs before the device is asked
for)."""
import os
import subprocess

import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFDRV = os.path.join(ROOT, "oracle", "_ref", "fm_refdrv")


@pytest.mark.skipif(not os.path.exists(REFDRV), reason="oracle A (compiled reference) not built")
@pytest.mark.parametrize("elem_type,n", [(mesh.TET4, 4), (mesh.HEXA8, 3)])
def test_element_arithmetic_bitwise_against_reference(tmp_path, elem_type, n):
    """formPoissonMatrix for every element and formPoissonSource for every
    ELSOURCE row (irSecondOrder), after FixedElementConnectivities, as the
    reference computes them: bit for bit."""
    p = mesh.poisson_box(n, elem_type=elem_type, seed=5)
    dat = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, dat)
    subprocess.run([REFDRV, dat, "poisson-elements", "--dump", str(tmp_path)], check=True, capture_output=True)
    raw = np.fromfile(str(tmp_path / "poisson_elements.f64"))
    E, npe = p.conn.shape
    conn = oracle_b.poisson_fix(p)
    Ka = raw[:E * npe * npe].reshape(E, npe, npe)
    fa = raw[E * npe * npe:].reshape(-1, npe)
    assert np.array_equal(Ka, oracle_b.poisson_elements(p, conn))
    assert np.array_equal(fa, oracle_b.poisson_sources(p, conn))


def test_fixed_connectivity_orientation():
    """The Kuhn tets of the cavity generator have positive volume in the VMS
    convention (x1-x0, x2-x0, x3-x0), which is negative for femTetra4's
    shape functions (node 3 is the local origin): the Poisson driver's
    FixedElementConnectivities swaps nodes 0 and 1 of every one."""
    p = mesh.poisson_box(3)
    conn = oracle_b.poisson_fix(p)
    assert np.array_equal(conn[:, [1, 0, 2, 3]], p.conn)
    h = mesh.poisson_box(3, elem_type=mesh.HEXA8)
    assert np.array_equal(oracle_b.poisson_fix(h), h.conn)


@pytest.mark.parametrize("problem", [mesh.POISSON_CLASSIC, mesh.POISSON_PPE])
def test_oracle_solution_satisfies_its_system(problem):
    p = mesh.poisson_box(4, problem=problem, seed=2, dirichlet=problem == mesh.POISSON_CLASSIC)
    K, b, _ = oracle_b.poisson_system(p)
    x, _ = oracle_b.poisson_solve(p)
    if problem == mesh.POISSON_CLASSIC:
        assert np.linalg.norm(K @ x - b) <= 1e-12 * np.linalg.norm(b)
        assert np.allclose(x[p.dir_node], p.dir_value, rtol=0, atol=1e-14)
    else:
        # pure Neumann: K x equals the zero-sum part of b, x has zero mean
        bb = b - b.mean()
        assert np.linalg.norm(K @ x - bb) <= 1e-10 * np.linalg.norm(bb)
        assert abs(x.mean()) <= 1e-14 * np.abs(x).max()


def test_poisson_create_rejects_bad_input_and_needs_a_device():
    p = mesh.poisson_box(2)
    bad = mesh.poisson_box(2)
    bad.conn = bad.conn.copy()
    bad.conn[0, 0] = bad.n_nodes
    with pytest.raises(api.FmError) as ei:
        api.GpuPoisson(bad)
    assert ei.value.code == api.FM_ERR_INVALID
    bad = mesh.poisson_box(2)
    bad.source_elem = bad.source_elem.copy()
    bad.source_elem[0] = bad.n_elems
    with pytest.raises(api.FmError) as ei:
        api.GpuPoisson(bad)
    assert ei.value.code == api.FM_ERR_INVALID
    # FACENEUMANN offsets: must start at >= 0 and increase
    for off0, off1 in ((-1, None), (None, 0)):
        bad = mesh.poisson_box(2)
        assert bad.neumann_value.size > 0
        bad.neumann_off = bad.neumann_off.copy()
        if off0 is not None:
            bad.neumann_off[0] = off0
        if off1 is not None:
            bad.neumann_off[1] = bad.neumann_off[0]
        with pytest.raises(api.FmError) as ei:
            api.GpuPoisson(bad)
        assert ei.value.code == api.FM_ERR_INVALID
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(api.FmError) as ei:
            api.GpuPoisson(p)
        assert ei.value.code == api.FM_ERR_NODEVICE


def test_poisson_read_dat_input_checks(tmp_path):
    """fm_poisson_read_dat parses the reference's keywords on the host; bad
    files are rejected before any device is asked for."""
    with pytest.raises(api.FmError) as ei:
        api.GpuPoisson.read_dat(str(tmp_path / "missing.dat"))
    assert ei.value.code == api.FM_ERR_IO
    p = mesh.poisson_box(2)
    good = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, good)
    txt = open(good).read()
    bad = str(tmp_path / "bad.dat")
    open(bad, "w").write(txt.replace("PROBLEM POISSON", "PROBLEM EXPLICITVMS"))
    with pytest.raises(api.FmError) as ei:
        api.GpuPoisson.read_dat(bad)
    assert ei.value.code == api.FM_ERR_INVALID
    lines = [ln for ln in txt.splitlines() if not ln.startswith("ELDIFF 1 ")]
    open(bad, "w").write("\n".join(lines) + "\n")
    with pytest.raises(api.FmError) as ei:
        api.GpuPoisson.read_dat(bad)
    assert ei.value.code == api.FM_ERR_INVALID
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(api.FmError) as ei:
            api.GpuPoisson.read_dat(good)
        assert ei.value.code == api.FM_ERR_NODEVICE


@pytest.mark.skipif(not os.path.exists(REFDRV), reason="oracle A (compiled reference) not built")
@pytest.mark.parametrize("elem_type", [mesh.TET4, mesh.HEXA8])
def test_wall_distance_bitwise_against_reference(tmp_path, elem_type):
    """evalDistanceFromPoissonSolution of the reference and the oracle's
    restatement on the same nodal solution: bit for bit."""
    p = mesh.poisson_box(4, elem_type=elem_type, problem=mesh.POISSON_DISTANCE, seed=13)
    dat = str(tmp_path / "p.dat")
    mesh.write_poisson_dat(p, dat)
    x, d = oracle_b.poisson_solve(p)
    sol = str(tmp_path / "sol.f64")
    x.astype(np.float64).tofile(sol)
    subprocess.run([REFDRV, dat, "poisson-elements", "--dump", str(tmp_path), "--sol", sol], check=True,
                   capture_output=True)
    raw = np.fromfile(str(tmp_path / "poisson_elements.f64"))
    E, npe = p.conn.shape
    skip = E * npe * npe + p.source_elem.size * npe
    da = raw[skip:]
    assert da.size == E
    assert np.array_equal(da, d, equal_nan=True)
