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


def test_ascii_writer_prints_percent_e(tmp_path):
    """Every number of the velocity and pressure sections is printf's "%e" of
    the value (checked against Python's correctly rounded %-formatting) over
    the whole exponent range, signed zeros, halfway cases and infinities."""
    p = mesh.cavity(4, seed=9, steps=2)
    rng = np.random.default_rng(11)
    init = rng.standard_normal((p.n_nodes, 4)) * 10.0 ** rng.integers(-307, 307, (p.n_nodes, 4))
    specials = [0.0, -0.0, 5e-324, -2.2250738585072014e-308, 1.7976931348623157e308, 0.5, 2.5e-7, 1234565.0,
                9.9999995, 999999.5, np.inf, -np.inf]
    init.ravel()[:len(specials)] = specials
    p.init_state = init
    g = api.GpuProblem(p)
    path = str(tmp_path / "a.vtk")
    g.write_vtk(path)
    g.close()
    lines = open(path).read().split("\n")
    k = lines.index("VECTORS velocity double") + 1
    for i in range(p.n_nodes):
        assert lines[k + i] == " ".join("%e" % v for v in init[i, :3]) + " ", (i, lines[k + i])
    k = lines.index("SCALARS pressure double 1") + 2
    for i in range(p.n_nodes):
        assert lines[k + i] == "%e " % init[i, 3], (i, lines[k + i])
