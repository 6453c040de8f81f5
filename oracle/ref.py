"""Runner for oracle A, the reference solver compiled by oracle/build_ref.sh.

Test infrastructure only (the checker, never the product).  It writes a
problem as a .dat file plus a raw initial-state file, runs
``oracle/_ref/fm_refdrv`` (femModel::ReadFromFEMTextFile followed by the
reference's femVMSExplicitFluidSolver::solve or femSUPGExplicitFluidSolver::solve,
src/main.cpp:788-806) and reads back the full-precision dumps its
ExportToVTKLegacy hook writes.
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFDRV = os.path.join(HERE, "_ref", "fm_refdrv")


def available() -> bool:
    return os.path.isfile(REFDRV) and os.access(REFDRV, os.X_OK)


def read_dump(path: str) -> dict:
    """Read one FMDUMP1 file -> {'time': t, label: array (nvals, ncomp)}."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"FMDUMP1\x00":
        raise ValueError(f"{path}: not an FMDUMP1 file")
    off = 8
    t = np.frombuffer(data, np.float64, 1, off)[0]
    off += 8
    nres = int(np.frombuffer(data, np.int32, 1, off)[0])
    off += 4
    out = {"time": float(t)}
    for _ in range(nres):
        label = data[off:off + 32].split(b"\x00")[0].decode()
        off += 32
        typ, nc = np.frombuffer(data, np.int32, 2, off)
        off += 8
        nv = int(np.frombuffer(data, np.int64, 1, off)[0])
        off += 8
        vals = np.frombuffer(data, np.float64, nv * int(nc), off).reshape(nv, int(nc)).copy()
        off += 8 * nv * int(nc)
        out[label] = vals
        out[label + ".type"] = int(typ)
    return out


def run(problem, workdir: str | None = None, solver: str | None = None, timing: bool = False,
        vtk: bool = False, timeout: float | None = None) -> dict:
    """Run the reference on ``problem``; return {step: dump dict} (+ timing).

    Output steps follow the reference's save counter: with TIMESTEP dt N s the
    solvers write steps s+1, 2s+1, ... (s >= 1) and step 1 only when s == 0,
    plus the initial state (step 0).
    """
    from femorph_b200.mesh import write_dat, VMS

    if not available():
        raise RuntimeError("oracle/_ref/fm_refdrv is missing; run oracle/build_ref.sh")
    own = workdir is None
    wd = tempfile.mkdtemp(prefix="fm_ref_") if own else workdir
    os.makedirs(wd, exist_ok=True)
    dat = os.path.join(wd, "model.dat")
    write_dat(problem, dat)
    args = [REFDRV, dat, solver or ("vms" if problem.solver == VMS else "supg"), "--dump", wd]
    if problem.init_state is not None:
        ic = os.path.join(wd, "ic.f64")
        np.ascontiguousarray(problem.init_state, np.float64).tofile(ic)
        args += ["--ic", ic, "4"]
    tpath = os.path.join(wd, "timing.txt")
    if timing:
        args += ["--timing", tpath]
    if vtk:
        args += ["--vtk"]
    r = subprocess.run(args, cwd=wd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"fm_refdrv failed ({r.returncode}): {r.stderr[-2000:]}\n{r.stdout[-2000:]}")
    out = {}
    for fn in os.listdir(wd):
        m = re.match(r".*_(\d+)\.vtk\.f64$", fn)
        if m:
            out[int(m.group(1))] = read_dump(os.path.join(wd, fn))
    if timing:
        out["timing"] = read_timing(tpath)
    out["stdout"] = r.stdout
    out["workdir"] = wd
    return out


def read_timing(path: str) -> dict:
    """Parse the driver's --timing file: parse time and BC-call timestamps."""
    parse = None
    stamps = []
    with open(path) as f:
        for line in f:
            if line.startswith("# parsed"):
                parse = float(line.split()[2])
            elif line.strip():
                a, b = line.split()
                stamps.append((float(a), float(b)))
    return {"parse_s": parse, "stamps": np.array(stamps).reshape(-1, 2)}
