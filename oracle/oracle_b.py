"""ctypes wrapper of oracle B (oracle/fm_oracle.c), the plain-C restatement.

Test infrastructure only: the checker used by tests/, smoke() and the
CPU-baseline leg of bench.py.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libfm_oracle.so")
_lib = None

_GLOB = {"NONE": 0, "X": 1, "Y": 2, "Z": 4, "XY": 3, "YZ": 6, "XZ": 5}


def build() -> str:
    src = os.path.join(HERE, "fm_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "_build/libfm_oracle.so"])
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.fmo_create.restype = P
        L.fmo_create.argtypes = [C.c_int64, C.c_int64, C.c_int, P, P, C.c_int, P, C.c_double, C.c_double, C.c_int,
                                 P, C.c_int, C.c_int, P, P, P, C.c_int, P, P, C.c_int, P, P, P]
        L.fmo_step.argtypes = [P, C.c_int]
        L.fmo_get.argtypes = [P, P, P, P, P]
        L.fmo_destroy.argtypes = [P]
        L.fmo_set_threads.argtypes = [C.c_int]
        L.fmo_get_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    """Host threads of the element loops (results do not depend on it)."""
    lib().fmo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().fmo_get_threads())


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class OracleSolve:
    """One CPU solve of ``problem`` (a femorph_b200.mesh.Problem)."""

    def __init__(self, p):
        L = lib()
        self.p = p
        self._keep = [
            np.ascontiguousarray(p.coords, np.float64), np.ascontiguousarray(p.conn, np.int32),
            np.ascontiguousarray(p.props, np.float64), np.ascontiguousarray(p.ex_opts, np.int32),
            np.ascontiguousarray(p.vel_node, np.int32), np.ascontiguousarray(p.vel_vals, np.float64).reshape(-1, 4),
            np.ascontiguousarray(p.vel_dir, np.int32), np.ascontiguousarray(p.dir_node, np.int32),
            np.ascontiguousarray(p.dir_vals, np.float64).reshape(-1, 3), np.ascontiguousarray(p.pres_node, np.int32),
            np.ascontiguousarray(p.pres_vals, np.float64),
            None if p.init_state is None else np.ascontiguousarray(p.init_state, np.float64)]
        x, conn, props, exo, vn, vv, vd, dn, dv, pn, pv, init = self._keep
        self.h = L.fmo_create(p.n_nodes, p.n_elems, p.elem_type, _ptr(x), _ptr(conn), p.solver, _ptr(props),
                              p.time_step, p.dual_step, p.tot_dual_steps, _ptr(exo), _GLOB[p.glob_fixed],
                              len(vn), _ptr(vn), _ptr(vv), _ptr(vd), len(dn), _ptr(dn), _ptr(dv),
                              len(pn), _ptr(pn), _ptr(pv), _ptr(init))

    def step(self, n: int = 1) -> None:
        err = lib().fmo_step(self.h, n)
        if err:
            raise RuntimeError(f"oracle B error {err}")

    def state(self):
        """(state (N,4), elem (E,3), extra, time) -- see fmo_get in fm_oracle.c."""
        p = self.p
        st = np.zeros((p.n_nodes, 4))
        el = np.zeros((p.n_elems, 3))
        ex = np.zeros((p.n_elems, 12)) if p.solver == 0 else np.zeros((p.n_nodes, 3))
        t = np.zeros(1)
        lib().fmo_get(self.h, _ptr(st), _ptr(el), _ptr(ex), _ptr(t))
        return st, el, ex, float(t[0])

    def close(self):
        if self.h:
            lib().fmo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
