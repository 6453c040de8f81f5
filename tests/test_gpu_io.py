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


def _read_vtu(path):
    """Arrays of a VTU file with raw appended data (UInt64 block sizes), by name."""
    import re
    data = open(path, "rb").read()
    start = data.index(b'<AppendedData encoding="raw">')
    base = data.index(b"_", start) + 1
    head = data[:start].decode()
    piece = re.search(r'NumberOfPoints="(\d+)" NumberOfCells="(\d+)"', head)
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="(\d+)")? '
                         r'format="appended" offset="(\d+)"/>', head):
        typ, name, comps, off = m.group(1), m.group(2) or "Points", int(m.group(3) or 1), int(m.group(4))
        n = int(np.frombuffer(data, np.uint64, 1, base + off)[0])
        dt = {"Float64": "<f8", "Int32": "<i4", "UInt8": "u1"}[typ]
        arr = np.frombuffer(data, dt, n // np.dtype(dt).itemsize, base + off + 8)
        out[name] = arr.reshape(-1, comps) if comps > 1 else arr
    return out, int(piece.group(1)), int(piece.group(2))


@pytest.mark.parametrize("case", ["vms", "supg_hexa"])
def test_vtu_holds_the_state_exactly(case):
    p = mesh.cavity(5, seed=6, steps=3) if case == "vms" else mesh.channel(6, 3, 3, seed=3, steps=3, noise=1e-3)
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.step(2)
    b.sync()
    path = os.path.join(tempfile.mkdtemp(), "s.vtu")
    g.write_vtu(path)
    V, n, e = _read_vtu(path)
    assert (n, e) == (p.n_nodes, p.n_elems)
    u, pe, el, _ = g.state()
    assert np.array_equal(V["velocity"], u) and np.array_equal(V["pressure"], pe)
    assert np.array_equal(V["Points"], p.coords)
    npe = p.elem_type
    assert np.array_equal(V["connectivity"].reshape(-1, npe), p.conn)
    assert np.array_equal(V["offsets"], npe * np.arange(1, p.n_elems + 1))
    assert np.all(V["types"] == (10 if npe == 4 else 12))
    if case == "vms":
        assert np.array_equal(V["subgrid_u"], el)
    else:
        assert np.array_equal(V["lambda"], el[:, 0]) and np.array_equal(V["regime"], el[:, 1])
    # the same BC markers as the legacy binary writer
    g.write_vtk(path + ".vtk", binary=True)
    Bn = _read_binary_vtk(path + ".vtk", p.n_nodes, p.n_elems)
    assert np.array_equal(V["dirBC"], Bn["dirBC"])
    b.close()
    g.close()
