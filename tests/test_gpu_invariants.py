"""Element-kinematics invariants: the asserted form of the checks the
reference's femTestSolver prints (src/femSolver.cpp:656-...; the reference
has no test suite of its own).

* The lumped masses sum to rho x the mesh volume (unit cube, 4 x 1 x 1
  channel), on the host.
* A linear field's gradient is exact, as the patch test of the SUPG viscous
  operator K2 (femSUPGExplicitFluidSolver.cpp:138-331): with the
  divergence-free linear velocity u = (y, z, x) prescribed on the boundary
  and as the initial state, the strain is the same constant in every element,
  so the assembled K2 u cancels at every interior node and one step leaves
  the interior nodes where they were.  This exercises the device Jacobians,
  inverses and global derivatives of tet4 and (jittered) hexa8 elements.
"""
import numpy as np
import pytest

from femorph_b200 import api, mesh


def test_lumped_masses_sum_to_volume():
    vms = mesh.cavity(6, seed=1)
    assert abs(api.GpuProblem(vms).mass().sum() - 1.0) < 1e-13
    # SUPG tet4: the reference's tet shape functions (femTetra4.cpp:295-330)
    # give the Kuhn tets, oriented for the VMS formulas, a negative Jacobian,
    # and form_lumped_mass keeps its sign (so does K: the update is the same)
    tet = mesh.cavity(5, seed=2, solver=mesh.SUPG, rho=2.0)
    m = api.GpuProblem(tet).mass().reshape(-1, 3)
    assert abs(abs(m[:, 0].sum()) - 2.0) < 1e-13
    hexa = mesh.channel(8, 4, 3, seed=3, rho=3.0)
    m = api.GpuProblem(hexa).mass().reshape(-1, 3)
    assert abs(m[:, 0].sum() - 3.0 * 4.0) < 1e-12


def _patch_problem(p):
    """p with K2 only (EXOPTS 1 0 0 1 0 0), u = (y, z, x) everywhere and held on
    the boundary."""
    X = np.asarray(p.coords)
    lin = np.stack([X[:, 1], X[:, 2], X[:, 0]], 1)
    lo, hi = X.min(0), X.max(0)
    bnd = np.any((X < lo + 1e-12) | (X > hi - 1e-12), axis=1)
    p.ex_opts = (1, 0, 0, 1, 0, 0)
    p.vel_node = np.zeros(0, np.int32)
    p.vel_vals = np.zeros((0, 4))
    p.vel_dir = np.zeros(0, np.int32)
    p.dir_node = np.nonzero(bnd)[0].astype(np.int32)
    p.dir_vals = lin[bnd]
    init = np.zeros((X.shape[0], 4))
    init[:, :3] = lin
    p.init_state = init
    return p, lin, ~bnd


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tet4", "hexa8"])
@pytest.mark.parametrize("precision,tol", [(api.FM_FP64, 1e-12), (api.FM_MIXED, 2e-6)])
def test_supg_viscous_patch_test(kind, precision, tol):
    if kind == "tet4":
        p = mesh.cavity(6, seed=4, solver=mesh.SUPG)
    else:
        p = mesh.channel(8, 4, 4, seed=5, jitter=0.2)
    p, lin, inner = _patch_problem(p)
    assert inner.sum() > 10
    g = api.GpuProblem(p, precision)
    b = api.Batch([g])
    b.step(1)
    b.sync()
    u, _, _, _ = g.state(elements=False)
    b.close()
    err = np.abs(u[inner] - lin[inner]).max() / np.abs(lin).max()
    assert err < tol, err
    # the boundary keeps its prescribed values exactly
    assert np.array_equal(u[~inner], lin[~inner])
