"""The writers on a problem that is not in a batch: they export the initial
state given at fm_problem_create (zeros without one) with zero element
fields, in the same three layouts as a placed problem's state (legacy ASCII
VTK, legacy binary VTK, VTU).  No GPU needed."""
import numpy as np
import pytest

from femorph_b200 import api, mesh
from test_gpu_io import _read_binary_vtk, _read_vtu, _sections


@pytest.mark.parametrize("case", ["vms", "supg_hexa", "no_init"])
def test_writers_export_the_initial_state_before_placement(tmp_path, case):
    p = mesh.channel(6, 3, 3, seed=3, steps=3, noise=1e-3) if case == "supg_hexa" else mesh.cavity(5, seed=6, steps=3)
    if case == "no_init":
        p.init_state = None
    init = np.zeros((p.n_nodes, 4)) if p.init_state is None else np.asarray(p.init_state, np.float64)
    assert case == "no_init" or np.abs(init[:, :3]).max() > 0
    vms = p.solver == mesh.VMS
    g = api.GpuProblem(p)
    g.write_vtu(str(tmp_path / "s.vtu"))
    g.write_vtk(str(tmp_path / "b.vtk"), binary=True)
    g.write_vtk(str(tmp_path / "a.vtk"))
    g.close()
    V, n, e = _read_vtu(str(tmp_path / "s.vtu"))
    assert (n, e) == (p.n_nodes, p.n_elems)
    assert np.array_equal(V["velocity"], init[:, :3]) and np.array_equal(V["Points"], p.coords)
    assert np.array_equal(V["connectivity"].reshape(-1, p.elem_type), p.conn)
    if vms:
        assert np.array_equal(V["pressure"], init[:, 3]) and not V["subgrid_u"].any()
    else:
        assert not V["pressure"].any() and not V["lambda"].any() and not V["regime"].any()
    Bn = _read_binary_vtk(str(tmp_path / "b.vtk"), p.n_nodes, p.n_elems)
    assert np.array_equal(Bn["velocity"].reshape(-1, 3), init[:, :3])
    assert np.array_equal(Bn["dirBC"], V["dirBC"]) and not Bn["normal"].any() and not Bn["neuBC"].any()
    A = _sections(str(tmp_path / "a.vtk"))
    assert np.allclose(np.array(A["VECTORS velocity"]), init[:, :3], rtol=2e-6, atol=1e-300)
    assert np.array_equal(np.array(A["SCALARS dirBC"]).ravel(), V["dirBC"])
    assert len(A["VECTORS normal"]) == p.n_elems and not np.array(A["VECTORS normal"]).any()
