"""The C ABI's VTK writer against the reference's own exporter (oracle A with
--vtk).  The VTK files
must agree line by line in layout and to the printed digits in value,
except res_v / res_p, the reference's diagnostic averages of a partially
assembled residual, which are written as zeros."""
import os
import tempfile

import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import ref

pytestmark = pytest.mark.gpu


def _sections(path):
    """{section header: [rows of floats]} in file order."""
    out, cur = {}, None
    for line in open(path):
        tok = line.split()
        if not tok:
            continue
        if tok[0] in ("POINTS", "CELLS", "CELL_TYPES", "VECTORS", "SCALARS", "POINT_DATA", "CELL_DATA"):
            cur = " ".join(tok[:2])
            out[cur] = []
            continue
        if tok[0] in ("LOOKUP_TABLE", "#", "Model", "ASCII", "DATASET"):
            continue
        if cur is not None:
            out[cur].append([float(x) for x in tok])
    return out


def test_vtk_writer_matches_reference_exporter():
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    p = mesh.cavity(4, seed=2, steps=3)
    p.save_every = 1
    wd = tempfile.mkdtemp()
    ref.run(p, workdir=wd, vtk=True)
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.step(3)
    b.sync()
    mine = os.path.join(wd, "mine.vtk")
    g.write_vtk(mine)
    A, G = _sections(os.path.join(wd, "out_Step_3.vtk")), _sections(mine)
    assert list(A) == list(G)
    for k in A:
        if "res_v" in k or "res_p" in k:
            continue
        a, gg = np.array(A[k]), np.array(G[k])
        assert a.shape == gg.shape, k
        if a.size == 0:
            continue
        if "subgrid" in k:
            # centroid averages of the Gauss-point subscales: zero up to rounding
            assert np.abs(gg - a).max() <= 1e-16, k
            continue
        # values at the rounding-noise level (|x| ~ 1e-16 of the field) compare absolutely
        assert np.allclose(gg, a, rtol=2e-6, atol=1e-13 * max(np.abs(a).max(), 1e-300)), k
    b.close()
    g.close()


def _read_binary_vtk(path, n_nodes, n_elems):
    """Sections of a legacy BINARY VTK file written by fm_problem_write_vtk_binary."""
    data = open(path, "rb").read()
    pos, out, n_data = 0, {}, n_nodes

    def line():
        nonlocal pos
        while data[pos:pos + 1] == b"\n":
            pos += 1
        end = data.index(b"\n", pos)
        s = data[pos:end].decode()
        pos = end + 1
        return s

    for _ in range(4):
        line()
    while pos < len(data) - 1:
        hdr = line().split()
        if hdr[0] == "POINT_DATA":
            n_data = n_nodes
            continue
        if hdr[0] == "CELL_DATA":
            n_data = n_elems
            continue
        if hdr[0] == "POINTS":
            key, dt, cnt = "POINTS", ">f4", 3 * int(hdr[1])
        elif hdr[0] == "CELLS":
            key, dt, cnt = "CELLS", ">i4", int(hdr[2])
        elif hdr[0] == "CELL_TYPES":
            key, dt, cnt = "CELL_TYPES", ">i4", int(hdr[1])
        else:
            key, dt = hdr[1], ">f8"
            cnt = 3 * n_data if hdr[0] == "VECTORS" else n_data
            if hdr[0] == "SCALARS":
                line()  # LOOKUP_TABLE default
        arr = np.frombuffer(data, dtype=dt, count=cnt, offset=pos)
        pos += arr.nbytes
        out[key] = arr
    return out


def test_binary_vtk_has_the_ascii_content():
    p = mesh.channel(6, 3, 3, seed=3, steps=3, noise=1e-3)
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.step(2)
    b.sync()
    wd = tempfile.mkdtemp()
    g.write_vtk(os.path.join(wd, "a.vtk"))
    g.write_vtk(os.path.join(wd, "b.vtk"), binary=True)
    A = _sections(os.path.join(wd, "a.vtk"))
    Bn = _read_binary_vtk(os.path.join(wd, "b.vtk"), p.n_nodes, p.n_elems)
    u, pe, el, _ = g.state()
    assert np.array_equal(Bn["velocity"].reshape(-1, 3), u)
    assert np.array_equal(Bn["pressure"], pe) and np.array_equal(Bn["lambda"], el[:, 0])
    assert np.array_equal(Bn["CELLS"].reshape(-1, 9)[:, 1:], p.conn)
    assert np.allclose(np.array(A["VECTORS velocity"]).ravel(), u.ravel(), rtol=2e-6, atol=1e-300)
    assert np.allclose(Bn["POINTS"].reshape(-1, 3), p.coords, rtol=1e-6)
    b.close()
    g.close()
