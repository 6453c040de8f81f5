"""Drop-in check: the reference's own driver path (femModel::ReadFromFEMTextFile
-> solver.solve(model) -> femModel::ExportToVTKLegacy) with the reference
solver classes (oracle/_ref/fm_refdrv) and with femorph_b200's femSolver
adapters (oracle/_ref/fm_gpudrv, the same objects plus
femorph_b200/adapter), compared step by step on the full-precision dumps of
every exported result."""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from femorph_b200 import mesh
from oracle import ref

pytestmark = pytest.mark.gpu
GPUDRV = os.path.join(os.path.dirname(ref.REFDRV), "fm_gpudrv")


def _run(binary, dat, solver, wd, stdout=False):
    os.makedirs(wd, exist_ok=True)
    r = subprocess.run([binary, dat, solver, "--dump", wd], cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    out = {}
    for fn in os.listdir(wd):
        if fn.endswith(".vtk.f64"):
            step = int(fn.split("_")[-1].split(".")[0])
            out[step] = ref.read_dump(os.path.join(wd, fn))
    return (out, r.stdout) if stdout else out


_VMS_ROW = re.compile(r"^\s*(\d+)\.(\d+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s*$")


def _vms_rows(text):
    """The VMS solver's per-dual-iteration lines: (step, dual, time, |res_u|, |res_p|, CFL)."""
    rows = []
    for line in text.splitlines():
        m = _VMS_ROW.match(line)
        if m:
            rows.append((int(m.group(1)), int(m.group(2))) + tuple(float(m.group(k)) for k in range(3, 7)))
    return rows


def _rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture
def workdir():
    d = tempfile.mkdtemp(prefix="fm_dropin_")
    yield d
    shutil.rmtree(d, ignore_errors=True)


def _need():
    if not (ref.available() and os.path.exists(GPUDRV)):
        pytest.skip("oracle/_ref binaries not built")


def test_dropin_vms(workdir):
    _need()
    p = mesh.cavity(5, seed=2, steps=6)
    p.init_state = None
    p.save_every = 2
    dat = os.path.join(workdir, "model.dat")
    mesh.write_dat(p, dat)
    A = _run(ref.REFDRV, dat, "vms", os.path.join(workdir, "ref"))
    G = _run(GPUDRV, dat, "vms-gpu", os.path.join(workdir, "gpu"))
    assert sorted(A) == sorted(G) == [0, 3, 5]
    for s in A:
        for lab in ("velocity", "pressure"):
            assert _rel(G[s][lab], A[s][lab]) <= 1e-12, (s, lab)
        if s > 0:
            # centroid average of the Gauss-point subscales: zero up to rounding
            # by construction of the orthogonal subscale, so checked absolutely
            assert np.abs(G[s]["subgrid_u"] - A[s]["subgrid_u"]).max() <= 1e-16


def test_dropin_vms_log_and_centroid_residuals(workdir):
    """The reference's per-dual-iteration log line (time, max centroid
    residual norms, CFL) and its res_v / res_p fields, rebuilt on the device
    from the iteration's element residuals as running sums in the
    reference's element order."""
    _need()
    p = mesh.cavity(5, seed=4, steps=5, lid=0.8)
    p.init_state = None
    p.tot_dual_steps = 1
    p.save_every = 2
    dat = os.path.join(workdir, "model.dat")
    mesh.write_dat(p, dat)
    A, out_a = _run(ref.REFDRV, dat, "vms", os.path.join(workdir, "ref"), stdout=True)
    G, out_g = _run(GPUDRV, dat, "vms-gpu", os.path.join(workdir, "gpu"), stdout=True)
    ra, rg = _vms_rows(out_a), _vms_rows(out_g)
    assert len(ra) == len(rg) == 5 * 2   # 5 steps of 2 dual iterations
    # the reference counts steps from 1, so its loopTime == 0 header never prints
    assert out_a.count("--- STARTING TIME LOOP") == out_g.count("--- STARTING TIME LOOP") == 0
    for a, g in zip(ra, rg):
        assert a[:2] == g[:2]
        assert abs(a[2] - g[2]) <= 1e-8, (a, g)
        for k in (3, 4):   # printed with 4 significant digits
            assert abs(a[k] - g[k]) <= 1e-3 * abs(a[k]) + 1e-300, (a, g)
        assert abs(a[5] - g[5]) <= 1.5e-3, (a, g)
    assert sorted(A) == sorted(G)
    for s in A:
        if s == 0:
            continue
        for lab in ("res_v", "res_p"):
            assert _rel(G[s][lab], A[s][lab]) <= 1e-9, (s, lab, _rel(G[s][lab], A[s][lab]))


def test_dropin_supg_hexa(workdir):
    _need()
    p = mesh.channel(6, 3, 3, seed=1, steps=5)
    p.init_state = None
    p.save_every = 1
    dat = os.path.join(workdir, "model.dat")
    mesh.write_dat(p, dat)
    A = _run(ref.REFDRV, dat, "supg", os.path.join(workdir, "ref"))
    G = _run(GPUDRV, dat, "supg-gpu", os.path.join(workdir, "gpu"))
    assert sorted(A) == sorted(G)
    for s in A:
        assert _rel(G[s]["velocity"], A[s]["velocity"]) <= 1e-12, s
        assert _rel(G[s]["pressure"], A[s]["pressure"]) <= 1e-11, s
        if s > 0:
            assert _rel(G[s]["lambda"], A[s]["lambda"]) <= 1e-11, s
            assert np.array_equal(G[s]["regime"], A[s]["regime"]), s
    # the per-step log (velocity extrema, tau / lambda / CFL / E / nu ranges,
    # reduced on the device) equals the reference's to its printed precision
    la = _log_rows(os.path.join(workdir, "ref", "log.txt"))
    lg = _log_rows(os.path.join(workdir, "gpu", "log.txt"))
    assert len(la) == len(lg) == 5
    for ra, rg in zip(la, lg):
        assert ra[0] == rg[0]
        for a, g in zip(ra[1:], rg[1:]):
            assert (np.isnan(a) and np.isnan(g)) or abs(a - g) <= 2e-3 * abs(a) + 1e-300, (ra, rg)


def _log_rows(path):
    rows = []
    for line in open(path):
        tok = line.split()
        if tok and tok[0].isdigit():
            rows.append([int(tok[0])] + [float(x) for x in tok[1:]])
    return rows
