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


# ---------------------------------------------------------------------------
# Poisson (femPoissonSolver::solve, femSolver.cpp:409-654)
# ---------------------------------------------------------------------------
def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


def poisson_fix(pp):
    """Connectivity after femModel::FixedElementConnectivities (a copy)."""
    L = lib()
    L.fmo_poisson_fix.restype = C.c_int64
    conn = np.ascontiguousarray(pp.conn, dtype=np.int32).copy()
    L.fmo_poisson_fix(C.c_int(conn.shape[1]), C.c_int64(conn.shape[0]), _vp(np.ascontiguousarray(pp.coords)),
                      _vp(conn))
    return conn


def poisson_elements(pp, conn):
    """femElement::formPoissonMatrix of every element: (E, npe, npe)."""
    E, npe = conn.shape
    K = np.empty((E, npe, npe))
    lib().fmo_poisson_elements(C.c_int(npe), C.c_int64(E), _vp(np.ascontiguousarray(pp.coords)), _vp(conn),
                               _vp(np.ascontiguousarray(pp.diffusivity)), _vp(K))
    return K


def poisson_sources(pp, conn):
    """femElement::formPoissonSource of every ELSOURCE row: (rows, npe)."""
    npe = conn.shape[1]
    out = np.empty((pp.source_elem.size, npe))
    se = np.ascontiguousarray(pp.source_elem, dtype=np.int32)
    sv = np.ascontiguousarray(pp.source_value, dtype=np.float64)
    lib().fmo_poisson_sources(C.c_int(npe), _vp(np.ascontiguousarray(pp.coords)), _vp(conn), C.c_int64(se.size),
                              _vp(se), _vp(sv), _vp(out))
    return out


def poisson_system(pp):
    """The reference's assembled system (femSolver.cpp:446-586): K (CSR) and
    the right-hand side after the sources, the face Neumann values and the
    Dirichlet rows (identity rows, value on the right-hand side).  Returns
    (K, b, fixed connectivity)."""
    import scipy.sparse as sp
    conn = poisson_fix(pp)
    E, npe = conn.shape
    N = pp.n_nodes
    Ke = poisson_elements(pp, conn)
    rows = np.repeat(conn, npe, axis=1).ravel()
    cols = np.tile(conn, (1, npe)).ravel()
    K = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(N, N)).tocsr()
    b = np.zeros(N)
    fs = poisson_sources(pp, conn)
    np.add.at(b, conn[pp.source_elem].ravel(), fs.ravel())  # rows in ELSOURCE order
    nv = np.zeros(N)
    cnt = np.diff(pp.neumann_off)
    share = np.repeat(pp.neumann_value / np.maximum(cnt, 1), cnt)
    np.add.at(nv, pp.neumann_nodes, share)
    b += nv
    if pp.dir_node.size:
        # identity rows (femTrilinosMatrix::applyBlockDirichelet), the last
        # NODEDIRBC row of a node wins (ReplaceGlobalValue)
        keep = np.ones(N, bool)
        keep[pp.dir_node] = False
        D = sp.diags(keep.astype(np.float64))
        K = (D @ K + sp.diags((~keep).astype(np.float64))).tocsr()
        K.eliminate_zeros()
        b[pp.dir_node] = pp.dir_value
    return K, b, conn


def poisson_solve(pp):
    """Direct solution of the reference's system (its Trilinos solve is not
    available here): x (the average subtracted for PPE) and, for DISTANCE,
    the element distances of evalDistanceFromPoissonSolution.  Without
    Dirichlet rows the system is singular: the right-hand side is reduced to
    its zero-sum part and node 0 is pinned, and the solution is compared up
    to a constant."""
    import scipy.sparse.linalg as spla
    K, b, conn = poisson_system(pp)
    if pp.dir_node.size == 0:
        import scipy.sparse as sp
        b = b - b.mean()
        keep = np.ones(K.shape[0])
        keep[0] = 0.0
        K = (sp.diags(keep) @ K + sp.diags(1.0 - keep)).tocsr()
        b[0] = 0.0
    x = spla.spsolve(K.tocsc(), b)
    if pp.problem == 1:
        x = x - x.mean()
    dist = None
    if pp.problem == 2:
        E, npe = conn.shape
        dist = np.empty(E)
        lib().fmo_poisson_distance(C.c_int(npe), C.c_int64(E), _vp(np.ascontiguousarray(pp.coords)), _vp(conn),
                                   _vp(np.ascontiguousarray(x)), _vp(dist))
    return x, dist
