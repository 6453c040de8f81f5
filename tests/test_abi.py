"""CPU checks of the C ABI: the library loads, exports every symbol the header
declares, validates inputs, and its host-side preparation (BC resolution,
lumped masses, .dat reader) matches the oracle without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from femorph_b200 import api, mesh
from oracle import oracle_b

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"FM_API\s+[\w\s\*]+?\b(fm_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = api.lib()
    syms = header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), s
    assert set(api.SYMBOLS) <= syms


def test_strerror_and_version():
    L = api.lib()
    assert L.fm_version() >= 100
    assert L.fm_strerror(api.FM_ERR_TABLE).decode().startswith("Could not find time")


def test_invalid_inputs_rejected():
    p = mesh.cavity(2, seed=0, steps=1)
    bad = mesh.cavity(2, seed=0, steps=1)
    bad.conn = bad.conn.copy()
    bad.conn[3, 2] = bad.n_nodes + 5
    with pytest.raises(api.FmError) as ei:
        api.GpuProblem(bad)
    assert ei.value.code == api.FM_ERR_INVALID
    hexa = mesh.channel(2, 2, 2, steps=1)
    hexa.solver = mesh.VMS
    with pytest.raises(api.FmError):
        api.GpuProblem(hexa)  # VMS is tet4-only
    tetb = mesh.cavity(2, seed=0, steps=1, solver=mesh.SUPG)
    tetb.ex_opts = (1, 1, 1, 1, 1, 1)
    with pytest.raises(api.FmError):
        api.GpuProblem(tetb)  # B-bar on tet4 reads out of bounds in the reference
    bd = mesh.cavity(2, seed=0, steps=1)
    bd.vel_dir = bd.vel_dir.copy()
    bd.vel_dir[0] = 9
    with pytest.raises(api.FmError):
        api.GpuProblem(bd)
    api.GpuProblem(p).close()


def test_masses_match_oracle_on_host():
    p = mesh.cavity(4, seed=3, steps=1)
    m = api.GpuProblem(p).mass()
    x, c = p.coords, p.conn
    V = np.linalg.det(np.stack([x[c[:, 1]] - x[c[:, 0]], x[c[:, 2]] - x[c[:, 0]], x[c[:, 3]] - x[c[:, 0]]], 1)) / 6
    ref = np.zeros(p.n_nodes)
    np.add.at(ref, c.ravel(), np.repeat(V / 4, 4))
    assert np.max(np.abs(m - ref)) <= 1e-15 * ref.max()
    q = mesh.channel(5, 3, 2, seed=1, steps=1)
    mq = api.GpuProblem(q).mass().reshape(-1, 3)
    _, _, lm, _ = oracle_b.OracleSolve(q).state()
    assert np.array_equal(mq, lm)


def test_dat_reader_round_trip(tmp_path):
    p = mesh.cavity(3, seed=4, steps=2)
    path = str(tmp_path / "m.dat")
    mesh.write_dat(p, path)
    h = C.c_void_p()
    api.check(api.lib().fm_problem_read_dat(path.encode(), 0, 0, C.byref(h)))
    nn, ne, et, sv = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
    api.check(api.lib().fm_problem_info(h, C.byref(nn), C.byref(ne), C.byref(et), C.byref(sv), None))
    assert (nn.value, ne.value, et.value, sv.value) == (p.n_nodes, p.n_elems, 4, 0)
    m = np.zeros(nn.value)
    api.check(api.lib().fm_problem_get_mass(h, m.ctypes.data))
    assert np.array_equal(m, api.GpuProblem(p).mass())
    api.lib().fm_problem_destroy(h)


def test_batch_without_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    g = api.GpuProblem(mesh.cavity(2, seed=0, steps=1))
    with pytest.raises(api.FmError) as ei:
        api.Batch([g])
    assert ei.value.code == api.FM_ERR_NODEVICE


def _mesh_struct(p, n_nodes=None, n_elems=None):
    keep = (np.ascontiguousarray(p.coords, np.float64), np.ascontiguousarray(p.conn, np.int32))
    m = api.FmMesh(p.elem_type, p.n_nodes if n_nodes is None else n_nodes,
                   p.n_elems if n_elems is None else n_elems, keep[0].ctypes.data, keep[1].ctypes.data)
    return m, keep


def test_edge_case_inputs_rejected():
    """Empty meshes, non-positive time steps, zero density, element types and
    tile sizes beyond the 16-bit tile-local indices are errors, not crashes."""
    L = api.lib()
    p = mesh.cavity(2, seed=0, steps=1)
    prm = api.FmParams()
    prm.solver, prm.precision, prm.time_step = p.solver, api.FM_FP64, p.time_step
    for i in range(5):
        prm.props[i] = float(p.props[i])
    h = C.c_void_p()
    for nn, ne in ((0, p.n_elems), (p.n_nodes, 0)):
        m, keep = _mesh_struct(p, nn, ne)
        assert L.fm_problem_create(C.byref(m), None, C.byref(prm), None, C.byref(h)) == api.FM_ERR_INVALID
    m, keep = _mesh_struct(p)
    m.elem_type = 6
    assert L.fm_problem_create(C.byref(m), None, C.byref(prm), None, C.byref(h)) == api.FM_ERR_INVALID
    m.elem_type = 4
    prm.time_step = 0.0
    assert L.fm_problem_create(C.byref(m), None, C.byref(prm), None, C.byref(h)) == api.FM_ERR_INVALID
    prm.time_step = p.time_step
    prm.props[0] = 0.0
    assert L.fm_problem_create(C.byref(m), None, C.byref(prm), None, C.byref(h)) == api.FM_ERR_INVALID
    prm.props[0] = 1.0
    assert L.fm_problem_create(C.byref(m), None, C.byref(prm), None, C.byref(h)) == api.FM_OK
    L.fm_problem_destroy(h)
    # tiles of more than 16383 tets overflow the 16-bit incidence entries
    # (reachable with the SUPG node cap of 4096 per tile)
    g = api.GpuProblem(mesh.cavity(16, seed=1, steps=1, solver=mesh.SUPG))
    with pytest.raises(api.FmError) as ei:
        g.prepare(tile_elems=20000, tile_nodes=4096)
    assert ei.value.code == api.FM_ERR_INVALID
    g.prepare()   # the default layout builds on the host without a GPU
    g.close()


def test_batch_composition_checked_before_device():
    """Problems of different solvers / precisions cannot share a batch."""
    a = api.GpuProblem(mesh.cavity(2, seed=0, steps=1))
    b = api.GpuProblem(mesh.cavity(2, seed=1, steps=1), api.FM_MIXED)
    arr = (C.c_void_p * 2)(a.h.value, b.h.value)
    h = C.c_void_p()
    assert api.lib().fm_batch_create(arr, 2, None, 0, C.byref(h)) == api.FM_ERR_INVALID
    a.close()
    b.close()


def test_capacity_bytes_grow_with_capacity_and_static_entry_validates():
    small = api.capacity_bytes(mesh.VMS, 4, 4, 100_000, 20_000, api.FM_FP64)
    big = api.capacity_bytes(mesh.VMS, 4, 4, 1_000_000, 200_000, api.FM_FP64)
    mixed = api.capacity_bytes(mesh.VMS, 4, 4, 1_000_000, 200_000, api.FM_MIXED)
    assert 0 < small < big and mixed < big
    # SUPG hexa8 pools hold the stored Gauss-point geometry: 8 points x 10
    # values an element, FP64 (640 B) or FP32 for the mixed form (320 B)
    E, N = 1_000_000, 1_100_000
    h64 = api.capacity_bytes(mesh.SUPG, 8, 1, E, N, api.FM_FP64)
    h32 = api.capacity_bytes(mesh.SUPG, 8, 1, E, N, api.FM_MIXED)
    assert h64 - h32 >= 320 * E
    assert h32 - api.capacity_bytes(mesh.SUPG, 4, 1, E, N, api.FM_MIXED) >= 320 * E
    # the allocation-free entry point checks its inputs before any device work
    L = api.lib()
    s = api.GpuProblem(mesh.cavity(2, seed=0, steps=1, solver=mesh.SUPG))
    s.prepare()
    assert L.fm_vms_solve_static(s.h, 1, 0, None, None, None) == api.FM_ERR_INVALID
    v = api.GpuProblem(mesh.cavity(2, seed=0, steps=1))
    assert L.fm_vms_solve_static(v.h, 1, 0, None, None, None) == api.FM_ERR_INVALID   # not prepared
    s.close()
    v.close()


def test_dat_reader_multi_block_file_equals_in_memory_problem(tmp_path):
    p = mesh.cavity(40, seed=3, steps=2)      # ~40 MB: several parse blocks
    path = str(tmp_path / "m.dat")
    mesh.write_dat(p, path)
    h = C.c_void_p()
    api.check(api.lib().fm_problem_read_dat(path.encode(), 0, 0, C.byref(h)))
    m = np.zeros(p.n_nodes)
    api.check(api.lib().fm_problem_get_mass(h, m.ctypes.data))
    assert np.array_equal(m, api.GpuProblem(p).mass())
    api.lib().fm_problem_destroy(h)


def test_checkpoint_needs_a_batch(tmp_path):
    """Checkpoint and restore refuse a problem outside a batch before any
    file or device access."""
    q = api.GpuProblem(mesh.cavity(2, seed=0, steps=1))
    path = str(tmp_path / "state.fmck")
    for f in (q.checkpoint, q.restore):
        with pytest.raises(api.FmError) as ei:
            f(path)
        assert ei.value.code == api.FM_ERR_INVALID
    assert not os.path.exists(path)
    q.close()


def test_unknown_register_budget_rejected_before_device():
    g = api.GpuProblem(mesh.cavity(2, seed=0, steps=1))
    for threads, ctas in ((128, 7), (256, 3), (128, 1)):
        with pytest.raises(api.FmError) as ei:
            api.Batch([g], threads=threads, ctas_per_sm=ctas)
        assert ei.value.code == api.FM_ERR_INVALID
    g.close()


def test_dat_reader_number_forms(tmp_path):
    """NODE coordinates written in the forms strtod accepts (leading '+',
    upper-case exponents, short decimals, leading zeros, tabs before the line
    end, comma separators, CRLF line ends, no final newline) read to the
    correctly rounded values: the lumped masses equal those of the same mesh
    built from the values parsed here (Python's float is correctly rounded
    like strtod)."""
    p = mesh.cavity(4, seed=8, steps=2)
    path = str(tmp_path / "m.dat")
    mesh.write_dat(p, path)
    forms = [lambda v: "+%.17e" % v if v >= 0 else "%.17e" % v, lambda v: "%.17E" % v, lambda v: "%.4f" % v,
             lambda v: "%.9g" % v, lambda v: ("0" + "%.12f" % v) if v >= 0 else "%.12f" % v]
    coords = np.array(p.coords, dtype=np.float64)
    out, k = [], 0
    for line in open(path).read().splitlines():
        t = line.split(" ")
        if t[0] == "NODE":
            i = int(t[1]) - 1
            txt = [forms[(k + c) % len(forms)](coords[i, c]) for c in range(3)]
            coords[i] = [float(x) for x in txt]
            sep = "," if k % 3 == 0 else " "
            line = sep.join(t[:2] + txt) + ("\t" if k % 4 == 1 else "")
            k += 1
        out.append(line + ("\r" if k % 5 == 2 else ""))
    with open(path, "w") as f:
        f.write("\n".join(out))
    h = C.c_void_p()
    api.check(api.lib().fm_problem_read_dat(path.encode(), 0, 0, C.byref(h)))
    m = np.zeros(p.n_nodes)
    api.check(api.lib().fm_problem_get_mass(h, m.ctypes.data))
    api.lib().fm_problem_destroy(h)
    q = mesh.cavity(4, seed=8, steps=2)
    q.coords = coords
    assert not np.array_equal(coords, np.asarray(p.coords))  # the short forms round some coordinates
    assert np.array_equal(m, api.GpuProblem(q).mass())


def test_autotune_cache_lookup_without_device(tmp_path):
    """fm_autotune answers from its cache file before it touches a device:
    the line whose key names the problem class (GPU model - "unknown" without
    a device -, solver, element type, precision, batch or single, log2 of the
    element count) gives the launch shape; a line written before the
    register budget was tuned (four fields) reads with ctas_per_sm 0; other
    lines are skipped.  Without a matching line and without a device the call
    fails loudly."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present (the key would name it)")
    except Exception:
        pass
    p = mesh.cavity(6, seed=1, steps=2)           # 1296 tets: 2^10 <= E < 2^11
    g = api.GpuProblem(p)
    cache = tmp_path / "tune.txt"
    key = "unknown/s0/e4/p0/n0/E2^10"
    cache.write_text("not a tuning line\nunknown/s0/e4/p1/n0/E2^10 256 128 128 5\n" + key + " 384 160 128 4\n")
    assert api.autotune([g], cache_path=str(cache)) == dict(tile_elems=384, tile_nodes=160, threads=128, ctas_per_sm=4)
    cache.write_text(key + " 512 256 256\n")
    assert api.autotune([g], cache_path=str(cache)) == dict(tile_elems=512, tile_nodes=256, threads=256, ctas_per_sm=0)
    cache.write_text("unknown/s0/e4/p0/n0/E2^11 512 256 128 3\n")
    with pytest.raises(api.FmError):
        api.autotune([g], cache_path=str(cache))
    g.close()
