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
