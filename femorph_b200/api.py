"""ctypes binding of the C ABI in include/femorph_b200.h.

The library is loaded from this package folder (built in-tree by
femorph_b200/build.py).  There is no fallback: if the shared library is
missing or no CUDA device is present, the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import mesh as _mesh

HERE = os.path.dirname(os.path.abspath(__file__))
# FEMORPH_B200_LIB selects another build of the library (e.g. a variant built
# elsewhere); by default the in-tree build is loaded.
LIB_PATH = os.environ.get("FEMORPH_B200_LIB") or os.path.join(HERE, "libfemorph_b200.so")

FM_OK, FM_ERR_INVALID, FM_ERR_OOM, FM_ERR_CUDA, FM_ERR_DIVERGED, FM_ERR_TIMEOUT, FM_ERR_TABLE, FM_ERR_IO, \
    FM_ERR_NODEVICE = range(9)
FM_FP64, FM_MIXED = 0, 1
_GLOB = {"NONE": 0, "X": 1, "Y": 2, "Z": 4, "XY": 3, "YZ": 6, "XZ": 5}

SYMBOLS = [
    "fm_strerror", "fm_last_error_message", "fm_version", "fm_problem_create", "fm_problem_destroy",
    "fm_problem_read_dat", "fm_problem_info", "fm_batch_create", "fm_batch_destroy", "fm_batch_step",
    "fm_batch_sync", "fm_batch_step_ragged", "fm_problem_get_state", "fm_problem_write_vtk",
    "fm_problem_get_mass", "fm_batch_last_timing", "fm_batch_estimate_bytes", "fm_batch_layout",
    "fm_batch_profile", "fm_autotune", "fm_batch_create_empty", "fm_batch_add", "fm_batch_remove",
    "fm_problem_prepare", "fm_batch_resident", "fm_batch_step_problems", "fm_problem_status",
    "fm_vms_solve_static", "fm_batch_capacity_bytes", "fm_problem_velocity_extrema", "fm_problem_supg_log_stats",
    "fm_partition_elements", "fm_problem_partition", "fm_problem_part_info", "fm_problem_part_map",
    "fm_problem_write_vtu", "fm_batch_exchange_account", "fm_batch_exchange_buffers", "fm_batch_exchange_begin",
    "fm_batch_exchange_end", "fm_batch_iterations_per_step", "fm_problem_checkpoint", "fm_problem_restore",
    "fm_batch_set_diagnostics", "fm_problem_vms_log", "fm_problem_vms_residuals",
    "fm_poisson_create", "fm_poisson_destroy", "fm_poisson_solve", "fm_poisson_get_solution", "fm_poisson_info", "fm_poisson_model",
    "fm_poisson_read_dat", "fm_poisson_write_vtk", "fm_problem_check_layout",
]

FM_POISSON_CLASSIC, FM_POISSON_PPE, FM_POISSON_DISTANCE = 0, 1, 2


class FmMesh(C.Structure):
    _fields_ = [("elem_type", C.c_int32), ("n_nodes", C.c_int64), ("n_elems", C.c_int64),
                ("coords", C.c_void_p), ("conn", C.c_void_p)]


class FmBC(C.Structure):
    _fields_ = [("n_vel_rows", C.c_int64), ("vel_node", C.c_void_p), ("vel_vals", C.c_void_p),
                ("vel_dir", C.c_void_p), ("n_dir", C.c_int64), ("dir_node", C.c_void_p), ("dir_vals", C.c_void_p),
                ("n_pres", C.c_int64), ("pres_node", C.c_void_p), ("pres_vals", C.c_void_p)]


class FmParams(C.Structure):
    _fields_ = [("solver", C.c_int32), ("precision", C.c_int32), ("props", C.c_double * 5),
                ("time_step", C.c_double), ("total_steps", C.c_int32), ("save_every", C.c_int32),
                ("dual_step", C.c_double), ("tot_dual_steps", C.c_int32), ("ex_opts", C.c_int32 * 6),
                ("glob_fixed", C.c_int32), ("exit_condition", C.c_double)]


class FmTuning(C.Structure):
    _fields_ = [("tile_elems", C.c_int32), ("tile_nodes", C.c_int32), ("threads", C.c_int32),
                ("graph_steps", C.c_int32), ("ctas_per_sm", C.c_int32), ("reserved", C.c_int32 * 3)]


class FmCapacity(C.Structure):
    _fields_ = [("solver", C.c_int32), ("elem_type", C.c_int32), ("precision", C.c_int32),
                ("max_problems", C.c_int32), ("max_elems", C.c_int64), ("max_nodes", C.c_int64),
                ("max_table_rows", C.c_int64), ("reserved", C.c_int64 * 4)]


class FmPoissonDesc(C.Structure):
    _fields_ = [("elem_type", C.c_int32), ("problem", C.c_int32), ("n_nodes", C.c_int64), ("n_elems", C.c_int64),
                ("coords", C.c_void_p), ("conn", C.c_void_p), ("diffusivity", C.c_void_p),
                ("n_sources", C.c_int64), ("source_elem", C.c_void_p), ("source_value", C.c_void_p),
                ("n_neumann", C.c_int64), ("neumann_off", C.c_void_p), ("neumann_nodes", C.c_void_p),
                ("neumann_value", C.c_void_p), ("n_dirichlet", C.c_int64), ("dir_node", C.c_void_p),
                ("dir_value", C.c_void_p)]


class FmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib():
    """Loads libfemorph_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m femorph_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.fm_strerror.restype = C.c_char_p
        L.fm_strerror.argtypes = [C.c_int]
        L.fm_last_error_message.restype = C.c_char_p
        L.fm_problem_create.argtypes = [P, P, P, P, P]
        L.fm_problem_destroy.argtypes = [P]
        L.fm_problem_read_dat.argtypes = [C.c_char_p, C.c_int32, C.c_int32, P]
        L.fm_problem_info.argtypes = [P, P, P, P, P, P]
        L.fm_batch_create.argtypes = [P, C.c_int32, P, C.c_int32, P]
        L.fm_batch_destroy.argtypes = [P]
        L.fm_batch_step.argtypes = [P, C.c_int32, P]
        L.fm_batch_sync.argtypes = [P]
        L.fm_batch_step_ragged.argtypes = [P, P, P]
        L.fm_problem_get_state.argtypes = [P, P, P, P, P]
        L.fm_problem_write_vtk.argtypes = [P, C.c_char_p]
        L.fm_problem_write_vtk_binary.argtypes = [P, C.c_char_p]
        L.fm_problem_write_vtu.argtypes = [P, C.c_char_p]
        L.fm_problem_checkpoint.argtypes = [P, C.c_char_p]
        L.fm_batch_set_diagnostics.argtypes = [P, C.c_int32]
        L.fm_batch_set_wait_limit.argtypes = [P, C.c_uint32]
        L.fm_math_check.argtypes = [P, C.c_int64, P]
        L.fm_problem_vms_log.argtypes = [P, P, C.c_int32, P]
        L.fm_problem_vms_residuals.argtypes = [P, P, P]
        L.fm_problem_restore.argtypes = [P, C.c_char_p]
        L.fm_problem_get_mass.argtypes = [P, P]
        L.fm_batch_last_timing.argtypes = [P, P, P]
        L.fm_batch_estimate_bytes.argtypes = [P, C.c_int32, P, P]
        L.fm_batch_layout.argtypes = [P, P, P, P, P]
        L.fm_batch_profile.argtypes = [P, C.c_int32, P, P]
        L.fm_autotune.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_char_p, P]
        L.fm_batch_create_empty.argtypes = [P, P, C.c_int32, P]
        L.fm_batch_add.argtypes = [P, P]
        L.fm_batch_remove.argtypes = [P, P]
        L.fm_problem_prepare.argtypes = [P, P]
        L.fm_batch_resident.argtypes = [P, P, P, P]
        L.fm_batch_step_problems.argtypes = [P, P, P, C.c_int32, P]
        L.fm_problem_status.argtypes = [P]
        L.fm_batch_capacity_bytes.argtypes = [P, P, P]
        L.fm_problem_velocity_extrema.argtypes = [P, P]
        L.fm_problem_supg_log_stats.argtypes = [P, P]
        L.fm_vms_solve_static.argtypes = [P, C.c_int32, C.c_int32, P, P, P]
        L.fm_partition_elements.argtypes = [P, C.c_int32, P]
        L.fm_problem_partition.argtypes = [P, P, C.c_int32, C.c_int32, P]
        L.fm_problem_part_info.argtypes = [P, P, P, P]
        L.fm_problem_part_map.argtypes = [P, P, P, P]
        L.fm_batch_exchange_buffers.argtypes = [P, P, P, P]
        L.fm_batch_exchange_begin.argtypes = [P, P]
        L.fm_batch_exchange_end.argtypes = [P, P]
        L.fm_batch_iterations_per_step.argtypes = [P, P]
        L.fm_batch_exchange_account.argtypes = [P, C.c_int32]
        L.fm_poisson_create.argtypes = [P, C.c_int32, P]
        L.fm_poisson_destroy.argtypes = [P]
        L.fm_poisson_solve.argtypes = [P, C.c_double, C.c_int32, P, P, P]
        L.fm_poisson_get_solution.argtypes = [P, P, P]
        L.fm_poisson_info.argtypes = [P, P, P]
        L.fm_poisson_model.argtypes = [P, P, P, P, P]
        L.fm_poisson_read_dat.argtypes = [C.c_char_p, C.c_int32, P]
        L.fm_problem_check_layout.argtypes = [P, P]
        L.fm_poisson_write_vtk.argtypes = [P, C.c_char_p]
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != FM_OK:
        L = lib()
        raise FmError(code, f"{L.fm_strerror(code).decode()}: {L.fm_last_error_message().decode()}")


def _p(a):
    return None if a is None or a.size == 0 else a.ctypes.data


class GpuProblem:
    """A femorph_b200 problem built from a femorph_b200.mesh.Problem."""

    def __init__(self, p: "_mesh.Problem", precision: int = FM_FP64):
        L = lib()
        self.src = p
        keep = dict(
            x=np.ascontiguousarray(p.coords, np.float64), conn=np.ascontiguousarray(p.conn, np.int32),
            vn=np.ascontiguousarray(p.vel_node, np.int32), vv=np.ascontiguousarray(p.vel_vals, np.float64).reshape(-1, 4),
            vd=np.ascontiguousarray(p.vel_dir, np.int32), dn=np.ascontiguousarray(p.dir_node, np.int32),
            dv=np.ascontiguousarray(p.dir_vals, np.float64).reshape(-1, 3),
            pn=np.ascontiguousarray(p.pres_node, np.int32), pv=np.ascontiguousarray(p.pres_vals, np.float64),
            init=None if p.init_state is None else np.ascontiguousarray(p.init_state, np.float64))
        m = FmMesh(p.elem_type, p.n_nodes, p.n_elems, _p(keep["x"]), _p(keep["conn"]))
        bc = FmBC(len(keep["vn"]), _p(keep["vn"]), _p(keep["vv"]), _p(keep["vd"]), len(keep["dn"]), _p(keep["dn"]),
                  _p(keep["dv"]), len(keep["pn"]), _p(keep["pn"]), _p(keep["pv"]))
        prm = FmParams()
        prm.solver = p.solver
        prm.precision = precision
        for i in range(5):
            prm.props[i] = float(p.props[i])
        prm.time_step = p.time_step
        prm.total_steps = p.total_steps
        prm.save_every = p.save_every
        prm.dual_step = p.dual_step
        prm.tot_dual_steps = p.tot_dual_steps
        for i in range(6):
            prm.ex_opts[i] = int(p.ex_opts[i])
        prm.glob_fixed = _GLOB[p.glob_fixed]
        prm.exit_condition = p.exit_condition
        h = C.c_void_p()
        check(L.fm_problem_create(C.byref(m), C.byref(bc), C.byref(prm), _p(keep["init"]) if keep["init"] is not None
                                  else None, C.byref(h)))
        self.h = h
        self.n_nodes, self.n_elems, self.solver = p.n_nodes, p.n_elems, p.solver

    def partition_elements(self, n_parts: int):
        """Default element split: part index of every element (Morton bands)."""
        out = np.zeros(self.n_elems, np.int32)
        check(lib().fm_partition_elements(self.h, int(n_parts), _p(out)))
        return out

    def part(self, n_parts: int, part: int, elem_part=None) -> "GpuPart":
        """The problem of one part of this mesh split into n_parts (elem_part:
        the part of every element, default Morton bands)."""
        ep = None if elem_part is None else np.ascontiguousarray(elem_part, np.int32)
        h = C.c_void_p()
        check(lib().fm_problem_partition(self.h, _p(ep), int(n_parts), int(part), C.byref(h)))
        return GpuPart(h, self.solver, self.src)

    def state(self, elements: bool = True):
        """(u (N,3), p (N,) VMS | (E,) SUPG, elem (E,3) VMS | (E,2) SUPG, sdus (E,12) VMS | None);
        elements=False reads velocity and pressure only (elem, sdus None)."""
        N, E = self.n_nodes, self.n_elems
        u = np.zeros((N, 3))
        vms = self.solver == _mesh.VMS
        p = np.zeros(N if vms else E)
        el = np.zeros((E, 3 if vms else 2)) if elements else None
        sd = np.zeros((E, 12)) if (vms and elements) else None
        check(lib().fm_problem_get_state(self.h, _p(u), _p(p), _p(el) if el is not None else None,
                                         _p(sd) if sd is not None else None))
        return u, p, el, sd

    def mass(self):
        m = np.zeros(self.n_nodes if self.solver == _mesh.VMS else self.n_nodes * 3)
        check(lib().fm_problem_get_mass(self.h, _p(m)))
        return m

    def write_vtk(self, path: str, binary: bool = False) -> None:
        f = lib().fm_problem_write_vtk_binary if binary else lib().fm_problem_write_vtk
        check(f(self.h, path.encode()))

    def write_vtu(self, path: str) -> None:
        """VTK XML UnstructuredGrid with raw appended binary arrays."""
        check(lib().fm_problem_write_vtu(self.h, path.encode()))

    def vms_log(self):
        """Queued VMS diagnostics rows (rows, 6): step, dual iteration, time,
        max centroid |res_u|, max |res_p|, CFL; the queue is emptied."""
        n = C.c_int32()
        check(lib().fm_problem_vms_log(self.h, None, 0, C.byref(n)))
        rows = np.zeros((n.value, 6))
        if n.value:
            check(lib().fm_problem_vms_log(self.h, _p(rows), n.value, C.byref(n)))
        return rows[: n.value]

    def vms_residuals(self):
        """Centroid residuals of the last recorded iteration: (res_u (E,3), res_p (E,))."""
        ru, rp = np.zeros((self.n_elems, 3)), np.zeros(self.n_elems)
        check(lib().fm_problem_vms_residuals(self.h, _p(ru), _p(rp)))
        return ru, rp

    def checkpoint(self, path: str) -> None:
        """Writes the problem's evolving state (it must sit in a batch) to a
        binary restart file."""
        check(lib().fm_problem_checkpoint(self.h, path.encode()))

    def restore(self, path: str) -> None:
        """Loads a restart file of this mesh and configuration into the
        problem (it must sit in a batch); stepping on continues that solve."""
        check(lib().fm_problem_restore(self.h, path.encode()))

    def check_layout(self, tile_elems=0, tile_nodes=0, threads=0) -> None:
        """Builds the tile layout for these sizes and checks its invariants
        (host only); raises FmError naming the first broken one."""
        t = FmTuning(tile_elems, tile_nodes, threads, 0, 0)
        check(lib().fm_problem_check_layout(self.h, C.byref(t)))

    def prepare(self, tile_elems=0, tile_nodes=0, threads=0) -> None:
        """Builds the tile layout now (host only, thread-safe per problem)."""
        t = FmTuning(tile_elems, tile_nodes, threads, 0)
        check(lib().fm_problem_prepare(self.h, C.byref(t)))

    def velocity_extrema(self):
        """(min u, max u, min v, max v, min w, max w, max |u|), reduced on the device."""
        out = np.zeros(7)
        check(lib().fm_problem_velocity_extrema(self.h, _p(out)))
        return out

    def supg_log_stats(self):
        """SUPG log quantities of the current state (see the C header)."""
        out = np.zeros(11)
        check(lib().fm_problem_supg_log_stats(self.h, _p(out)))
        return out

    def status(self) -> int:
        """Device status code of this problem in its batch (FM_OK when healthy)."""
        return lib().fm_problem_status(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().fm_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuPart(GpuProblem):
    """One part of a partitioned mesh (GpuProblem.part).  State and masses
    are in the part's local numbering; node_global / elem_global map them to
    the whole mesh, xidx gives each local node's exchange index (-1: not
    shared)."""

    def __init__(self, h, solver, src):
        L = lib()
        self.h = h
        self.src = src
        self.solver = solver
        nn, ne = C.c_int64(), C.c_int64()
        check(L.fm_problem_info(h, C.byref(nn), C.byref(ne), None, None, None))
        self.n_nodes, self.n_elems = nn.value, ne.value
        part, nparts, xt = C.c_int32(), C.c_int32(), C.c_int64()
        check(L.fm_problem_part_info(h, C.byref(part), C.byref(nparts), C.byref(xt)))
        self.part_index, self.n_parts, self.x_total = part.value, nparts.value, xt.value
        self.node_global = np.zeros(self.n_nodes, np.int32)
        self.elem_global = np.zeros(self.n_elems, np.int32)
        self.xidx = np.zeros(self.n_nodes, np.int32)
        check(L.fm_problem_part_map(h, _p(self.node_global), _p(self.elem_global), _p(self.xidx)))


class _DeviceArray:
    """A device buffer of the library seen through __cuda_array_interface__
    (torch.as_tensor wraps it without a copy)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 2, "strides": None}


class Batch:
    """Device-resident batch of GpuProblems (all share solver and element type)."""

    def __init__(self, problems, tile_elems=0, tile_nodes=0, threads=0, graph_steps=0, device=0, ctas_per_sm=0):
        L = lib()
        self.problems = list(problems)
        arr = (C.c_void_p * len(self.problems))(*[q.h.value for q in self.problems])
        t = FmTuning(tile_elems, tile_nodes, threads, graph_steps, ctas_per_sm)
        h = C.c_void_p()
        check(L.fm_batch_create(arr, len(self.problems), C.byref(t), device, C.byref(h)))
        self.h = h

    def step(self, n: int = 1, stream=None) -> None:
        check(lib().fm_batch_step(self.h, int(n), stream))

    def set_wait_limit(self, polls: int) -> None:
        """Polls of the VMS tile kernel's bounded chunk waits before FM_ERR_TIMEOUT."""
        check(lib().fm_batch_set_wait_limit(self.h, int(polls)))

    def set_diagnostics(self, enable: bool = True) -> None:
        """VMS: record the reference's log row and centroid residuals every
        dual iteration (GpuProblem.vms_log / vms_residuals)."""
        check(lib().fm_batch_set_diagnostics(self.h, 1 if enable else 0))

    def step_ragged(self, steps, stream=None) -> None:
        a = np.ascontiguousarray(steps, np.int32)
        check(lib().fm_batch_step_ragged(self.h, _p(a), stream))

    def sync(self) -> None:
        check(lib().fm_batch_sync(self.h))

    def last_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        check(lib().fm_batch_last_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def profile(self, n: int):
        """Runs n steps with per-kernel CUDA events: ({'tile': ms, 'iface': ms}, launches per kernel)."""
        ms = (C.c_double * 2)()
        ln = (C.c_int64 * 2)()
        check(lib().fm_batch_profile(self.h, int(n), ms, ln))
        return {"tile": ms[0], "iface": ms[1]}, ln[0]

    def exchange_buffers(self):
        """(send, recv, count) of a batch of partition parts: objects with
        __cuda_array_interface__ over count doubles each."""
        s, r, n = C.c_void_p(), C.c_void_p(), C.c_int64()
        check(lib().fm_batch_exchange_buffers(self.h, C.byref(s), C.byref(r), C.byref(n)))
        return _DeviceArray(s.value, n.value), _DeviceArray(r.value, n.value), n.value

    def exchange_begin(self, stream=None) -> None:
        check(lib().fm_batch_exchange_begin(self.h, stream))

    def exchange_end(self, stream=None) -> None:
        check(lib().fm_batch_exchange_end(self.h, stream))

    def exchange_account(self, iterations: int) -> None:
        """Counts iterations run by replaying captured begin/end pairs."""
        check(lib().fm_batch_exchange_account(self.h, int(iterations)))

    def iterations_per_step(self) -> int:
        n = C.c_int32()
        check(lib().fm_batch_iterations_per_step(self.h, C.byref(n)))
        return n.value

    def layout(self):
        a, b, c, d = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
        check(lib().fm_batch_layout(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return dict(tiles=a.value, iface_nodes=b.value, max_colors=c.value, slots=d.value)

    def close(self):
        if getattr(self, "h", None):
            lib().fm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def capacity_bytes(solver, elem_type, max_problems, max_elems, max_nodes, precision=FM_FP64, max_table_rows=0,
                   tile_elems=0, tile_nodes=0, threads=0) -> int:
    """Device bytes a Pool of these capacities allocates."""
    cap = FmCapacity(solver, elem_type, precision, max_problems, max_elems, max_nodes, max_table_rows)
    t = FmTuning(tile_elems, tile_nodes, threads, 0)
    out = C.c_int64()
    check(lib().fm_batch_capacity_bytes(C.byref(cap), C.byref(t), C.byref(out)))
    return out.value


class Pool:
    """Batch with fixed device pools that problems join and leave between
    launches (continuous batching)."""

    def __init__(self, solver, elem_type, max_problems, max_elems, max_nodes, precision=FM_FP64,
                 max_table_rows=0, tile_elems=0, tile_nodes=0, threads=0, graph_steps=0, device=0, ctas_per_sm=0):
        cap = FmCapacity(solver, elem_type, precision, max_problems, max_elems, max_nodes, max_table_rows)
        t = FmTuning(tile_elems, tile_nodes, threads, graph_steps, ctas_per_sm)
        h = C.c_void_p()
        check(lib().fm_batch_create_empty(C.byref(cap), C.byref(t), device, C.byref(h)))
        self.h = h
        self.members = []

    def add(self, q: GpuProblem) -> bool:
        """Places q; False when the pools have no room for it."""
        r = lib().fm_batch_add(self.h, q.h)
        if r == FM_ERR_OOM:
            return False
        check(r)
        self.members.append(q)
        return True

    def remove(self, q: GpuProblem) -> None:
        check(lib().fm_batch_remove(self.h, q.h))
        self.members.remove(q)

    def step(self, problems, steps, stream=None) -> None:
        """Advances each listed problem by its entry of `steps` (others idle)."""
        arr = (C.c_void_p * len(problems))(*[q.h.value for q in problems])
        a = np.ascontiguousarray(steps, np.int32)
        check(lib().fm_batch_step_problems(self.h, arr, _p(a), len(problems), stream))

    def sync(self) -> None:
        check(lib().fm_batch_sync(self.h))

    def wait(self) -> bool:
        """Waits for the pool's work; True when some resident problem reports
        a device error (FM_ERR_DIVERGED, FM_ERR_TABLE, FM_ERR_TIMEOUT), which
        GpuProblem.status() then tells apart; other errors raise."""
        r = lib().fm_batch_sync(self.h)
        if r in (FM_ERR_DIVERGED, FM_ERR_TABLE, FM_ERR_TIMEOUT):
            return True
        check(r)
        return False

    def last_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        check(lib().fm_batch_last_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def resident(self):
        a, b, c = C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().fm_batch_resident(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(problems=a.value, elems=b.value, largest_free_elems=c.value)

    def close(self):
        if getattr(self, "h", None):
            lib().fm_batch_destroy(self.h)
            self.h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(problems, device: int = 0, steps: int = 10, cache_path: str | None = None) -> dict:
    """Runs the library's autotuner on GpuProblems (not in a batch); returns
    the best launch shape as Batch keyword arguments."""
    arr = (C.c_void_p * len(problems))(*[q.h.value for q in problems])
    t = FmTuning()
    check(lib().fm_autotune(arr, len(problems), device, steps, cache_path.encode() if cache_path else None,
                            C.byref(t)))
    return dict(tile_elems=t.tile_elems, tile_nodes=t.tile_nodes, threads=t.threads, ctas_per_sm=t.ctas_per_sm)


def solve(p: "_mesh.Problem", steps: int | None = None, precision: int = FM_FP64, **tuning):
    """Convenience: one problem, `steps` time steps, returns GpuProblem + Batch."""
    gp = GpuProblem(p, precision)
    b = Batch([gp], **tuning)
    b.step(p.steps if steps is None else steps)
    b.sync()
    return gp, b


class GpuPoisson:
    """femPoissonSolver::solve (femSolver.cpp:409-654) on the GPU: the system
    of a `mesh.PoissonProblem` assembled on the host, solved by conjugate
    gradients on `device`."""

    def __init__(self, pp: "_mesh.PoissonProblem | None", device: int = 0, path: str | None = None):
        if pp is None:  # from a .dat file (fm_poisson_read_dat)
            h = C.c_void_p()
            check(lib().fm_poisson_read_dat(str(path).encode(), int(device), C.byref(h)))
            self.h = h
            self.n_nodes, self.n_elems, _, self.problem = self.model()
            return
        self._keep = [np.ascontiguousarray(a) for a in (
            pp.coords, pp.conn, pp.diffusivity, pp.source_elem, pp.source_value, pp.neumann_off, pp.neumann_nodes,
            pp.neumann_value, pp.dir_node, pp.dir_value)]
        co, cn, df, se, sv, no, nn, nv, dn, dv = self._keep
        d = FmPoissonDesc(int(cn.shape[1]), int(pp.problem), int(co.shape[0]), int(cn.shape[0]), _p(co), _p(cn), _p(df),
                          int(se.size), _p(se), _p(sv), int(nv.size), _p(no), _p(nn), _p(nv), int(dn.size), _p(dn),
                          _p(dv))
        h = C.c_void_p()
        check(lib().fm_poisson_create(C.byref(d), int(device), C.byref(h)))
        self.h = h
        self.n_nodes, self.n_elems, self.problem = int(co.shape[0]), int(cn.shape[0]), int(pp.problem)

    def solve(self, rel_tol: float = 1e-12, max_iter: int = 20000):
        """Returns (iterations, relative residual, device ms)."""
        it, rr, ms = C.c_int32(), C.c_double(), C.c_double()
        check(lib().fm_poisson_solve(self.h, float(rel_tol), int(max_iter), C.byref(it), C.byref(rr), C.byref(ms)))
        return int(it.value), float(rr.value), float(ms.value)

    @classmethod
    def read_dat(cls, path: str, device: int = 0):
        """The solver of a .dat file's Poisson model (fm_poisson_read_dat)."""
        return cls(None, device, path)

    def model(self):
        """(nodes, elements, element type, FM_POISSON_* problem) of the model."""
        n, e, t, pb = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        check(lib().fm_poisson_model(self.h, C.byref(n), C.byref(e), C.byref(t), C.byref(pb)))
        return int(n.value), int(e.value), int(t.value), int(pb.value)

    def solution(self):
        """(x, cell distance or None)."""
        x = np.empty(self.n_nodes)
        dist = np.empty(self.n_elems) if self.problem == FM_POISSON_DISTANCE else None
        check(lib().fm_poisson_get_solution(self.h, _p(x), _p(dist)))
        return x, dist

    def write_vtk(self, path: str) -> None:
        """The results in the reference exporter's legacy-VTK layout."""
        check(lib().fm_poisson_write_vtk(self.h, str(path).encode()))

    def info(self):
        r, z = C.c_int64(), C.c_int64()
        check(lib().fm_poisson_info(self.h, C.byref(r), C.byref(z)))
        return int(r.value), int(z.value)

    def close(self):
        if getattr(self, "h", None):
            lib().fm_poisson_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
