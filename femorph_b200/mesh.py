"""Seeded synthetic flow problems and the feMorph ``.dat`` text format.

The generators build the meshes, boundary conditions and initial states of the
explicit-flow workloads:

* ``cavity(n, ...)``   lid-driven cavity: unit cube, n^3 cells, each cut into 6
  tet4 by Kuhn subdivision along the (0,0,0)-(1,1,1) diagonal, interior nodes
  jittered by a seeded uniform +-0.1h, lid u=(U,0,0) on z=1, no-slip on the
  other faces, pressure pinned at node 0.
* ``channel(nx, ny, nz, ...)``  hexa8 channel on [0,4]x[0,1]x[0,1] with a
  parabolic inlet at x=0 (peak 1), no-slip walls and a free outlet.

``write_dat`` writes the keyword file read by the reference's
``femModel::ReadFromFEMTextFile`` (src/femModel.cpp:3719-4213): 1-based node
and element numbers, ``NODEVEL node vx vy vz t [dir]``, ``NODEDIRBC node vx vy
vz``, ``NODEPRES node p``, ``TIMESTEP dt totalSteps saveEvery``, ``DUALSTEP ds
nDual``, ``VMSPROPS rho mu invEps|alpha c1|cI c2``, ``EXOPTS``, ``NODEDOF``,
``OUTPUT``, ``LOGFILE``, ``EXITCOND``.  Coordinates and parameters are written
with 17 significant digits, so the values the reference parses with ``atof``
are bit-identical to the arrays handed to the GPU solver.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field

import numpy as np

TET4 = 4
HEXA8 = 8

VMS = 0
SUPG = 1


@dataclass
class Problem:
    """One explicit-flow solve: mesh, boundary conditions, parameters, state."""

    coords: np.ndarray                # (N, 3) float64
    conn: np.ndarray                  # (E, 4|8) int32, 0-based
    solver: int = VMS                 # VMS or SUPG
    props: tuple = (1.0, 0.01, 400.0, 4.0, 2.0)   # VMSPROPS
    time_step: float = 1e-3
    total_steps: int = 2              # TIMESTEP 2nd field: executes total_steps-1 steps
    save_every: int = 1000000
    dual_step: float = 1e-3
    tot_dual_steps: int = 0
    ex_opts: tuple = (1, 0, 1, 1, 1, 1)           # EXOPTS (SUPG)
    glob_fixed: str = "NONE"                       # NODEDOF fixed dofs (SUPG)
    exit_condition: float = 1.0e5
    max_node_dofs: int = 4
    # NODEVEL rows in file order: node, (vx, vy, vz, t), dir
    vel_node: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    vel_vals: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    vel_dir: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    # NODEDIRBC rows
    dir_node: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    dir_vals: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    # NODEPRES rows
    pres_node: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    pres_vals: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # initial nodal state before BCs, (N, 4): u, v, w, p
    init_state: np.ndarray | None = None
    name: str = ""

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def elem_type(self) -> int:
        return int(self.conn.shape[1])

    @property
    def steps(self) -> int:
        """Number of time steps the reference executes (TIMESTEP N runs N-1)."""
        return self.total_steps - 1


def _tet_volumes(coords: np.ndarray, conn: np.ndarray) -> np.ndarray:
    x0 = coords[conn[:, 0]]
    j = np.stack([coords[conn[:, 1]] - x0, coords[conn[:, 2]] - x0, coords[conn[:, 3]] - x0], axis=1)
    return np.linalg.det(j) / 6.0


def kuhn_cavity_mesh(n: int, seed: int, jitter: float = 0.1):
    """Unit cube, n^3 cells x 6 Kuhn tets, seeded interior jitter (+-jitter*h).

    Returns (coords, conn).  Tets are ordered cell-major (i, j, k lexicographic)
    and, within a cell, by the permutation order of the axes (0,1,2), (0,2,1),
    (1,0,2), (1,2,0), (2,0,1), (2,1,0); each tet is the path v, v+e_a,
    v+e_a+e_b, v+(1,1,1).  Nodes 0 and 1 are swapped where the Jacobian
    determinant is negative, because the reference's VMS solver takes
    V = detJ/6 without an absolute value (src/femVMSExplicitFluidSolver.cpp:73).
    """
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    idx = np.arange(n + 1, dtype=np.float64)
    X = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), -1).reshape(-1, 3) * h
    interior = np.all((X > 1e-12) & (X < 1.0 - 1e-12), axis=1)
    X[interior] += rng.uniform(-jitter * h, jitter * h, (int(interior.sum()), 3))
    ci, cj, ck = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    cells = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], 1).astype(np.int64)
    m = n + 1
    nid = lambda v: (v[:, 0] * m + v[:, 1]) * m + v[:, 2]
    tets = np.empty((cells.shape[0], 6, 4), np.int64)
    for p_i, perm in enumerate(itertools.permutations(range(3))):
        v = cells.copy()
        tets[:, p_i, 0] = nid(v)
        for s, ax in enumerate(perm):
            v = v.copy()
            v[:, ax] += 1
            tets[:, p_i, s + 1] = nid(v)
    conn = tets.reshape(-1, 4)
    vol = _tet_volumes(X, conn)
    neg = vol < 0
    conn[neg, 0], conn[neg, 1] = conn[neg, 1].copy(), conn[neg, 0].copy()
    return X, conn.astype(np.int32), rng


def cavity(n: int, seed: int = 0, lid: float = 1.0, mu: float = 0.01, rho: float = 1.0,
           inv_eps: float = 400.0, c1: float = 4.0, c2: float = 2.0, steps: int = 200,
           cfl: float = 0.2, solver: int = VMS, alpha: float = 1.0, c_i: float = 4.0,
           noise: float = 1e-3, dt: float | None = None) -> Problem:
    """Lid-driven cavity on the Kuhn-tet cube (VMS by default, SUPG optional).

    dt = cfl * h_min / (lid + sqrt(invEps)) with h_min = min cbrt(6V) for VMS:
    the artificial sound speed sqrt(invEps) must enter the explicit limit or the
    reference itself diverges.  Initial state: u = seeded uniform +-noise on
    every node (the BCs then overwrite boundary nodes), p = 0.
    """
    X, conn, rng = kuhn_cavity_mesh(n, seed)
    N = X.shape[0]
    init = np.zeros((N, 4))
    init[:, :3] = rng.uniform(-noise, noise, (N, 3))
    lid_nodes = np.nonzero(X[:, 2] > 1.0 - 1e-12)[0].astype(np.int32)
    on_bnd = np.any((X < 1e-12) | (X > 1.0 - 1e-12), axis=1)
    wall_nodes = np.nonzero(on_bnd & ~(X[:, 2] > 1.0 - 1e-12))[0].astype(np.int32)
    vol = _tet_volumes(X, conn)
    hmin = float(np.cbrt(6.0 * vol).min())
    if solver == VMS:
        props = (rho, mu, inv_eps, c1, c2)
        if dt is None:
            dt = cfl * hmin / (lid + math.sqrt(inv_eps))
        pres_node = np.array([0], np.int32)
        pres_vals = np.array([0.0])
        max_dofs = 4
    else:
        props = (rho, mu, alpha, c_i, 0.0)
        if dt is None:
            dt = min(cfl * hmin / lid, 0.1 * hmin * hmin * rho / mu)
        pres_node = np.zeros(0, np.int32)
        pres_vals = np.zeros(0)
        max_dofs = 3
    vel_vals = np.zeros((lid_nodes.size, 4))
    vel_vals[:, 0] = lid
    return Problem(
        coords=X, conn=conn, solver=solver, props=props, time_step=float(dt),
        total_steps=steps + 1, dual_step=float(dt), tot_dual_steps=0,
        max_node_dofs=max_dofs,
        vel_node=lid_nodes, vel_vals=vel_vals, vel_dir=np.full(lid_nodes.size, 6, np.int32),
        dir_node=wall_nodes, dir_vals=np.zeros((wall_nodes.size, 3)),
        pres_node=pres_node, pres_vals=pres_vals, init_state=init,
        name=f"cavity{n}_s{seed}")


def channel(nx: int = 256, ny: int = 64, nz: int = 64, seed: int = 0, mu: float = 0.005,
            rho: float = 1.0, steps: int = 500, alpha: float = 1.0, c_i: float = 4.0,
            jitter: float = 0.05, cfl: float = 0.2, dt: float | None = None,
            ex_opts=(1, 0, 1, 1, 1, 1), noise: float = 0.0) -> Problem:
    """Hexa8 channel [0,4]x[0,1]^2, parabolic inlet 16 y(1-y) z(1-z), SUPG.

    Hexa8 connectivity follows the reference's femHexa8 corner order
    (src/femHexa8.cpp:13-42): (0,0,0) (1,0,0) (1,1,0) (0,1,0) and the same at
    z+1.  Walls (y or z on the boundary, x > 0) are no-slip; the outlet x=4 is
    free (natural zero traction).
    """
    rng = np.random.default_rng(seed)
    L = np.array([4.0, 1.0, 1.0])
    h = L / np.array([nx, ny, nz])
    ii = [np.arange(m + 1, dtype=np.float64) for m in (nx, ny, nz)]
    X = np.stack(np.meshgrid(*ii, indexing="ij"), -1).reshape(-1, 3) * h
    tol = 1e-12
    inter = ((X[:, 0] > tol) & (X[:, 0] < L[0] - tol) & (X[:, 1] > tol) & (X[:, 1] < 1 - tol)
             & (X[:, 2] > tol) & (X[:, 2] < 1 - tol))
    X[inter] += rng.uniform(-jitter, jitter, (int(inter.sum()), 3)) * h
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = ci.ravel(), cj.ravel(), ck.ravel()
    nid = lambda a, b, c: (a * (ny + 1) + b) * (nz + 1) + c
    conn = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                     nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                     nid(i, j + 1, k + 1)], 1).astype(np.int32)
    N = X.shape[0]
    init = np.zeros((N, 4))
    if noise > 0:
        init[:, :3] = rng.uniform(-noise, noise, (N, 3))
    inlet = np.nonzero(X[:, 0] < tol)[0].astype(np.int32)
    y, z = X[inlet, 1], X[inlet, 2]
    vel_vals = np.zeros((inlet.size, 4))
    vel_vals[:, 0] = 16.0 * y * (1 - y) * z * (1 - z)
    walls = np.nonzero((X[:, 0] > tol) & ((X[:, 1] < tol) | (X[:, 1] > 1 - tol)
                                          | (X[:, 2] < tol) | (X[:, 2] > 1 - tol)))[0].astype(np.int32)
    hmin = float(h.min())
    if dt is None:
        dt = min(cfl * hmin / 1.0, 0.1 * hmin * hmin * rho / mu)
    return Problem(
        coords=X, conn=conn, solver=SUPG, props=(rho, mu, alpha, c_i, 0.0), time_step=float(dt),
        total_steps=steps + 1, dual_step=float(dt), max_node_dofs=3, ex_opts=tuple(ex_opts),
        vel_node=inlet, vel_vals=vel_vals, vel_dir=np.full(inlet.size, 6, np.int32),
        dir_node=walls, dir_vals=np.zeros((walls.size, 3)), init_state=init,
        name=f"channel{nx}x{ny}x{nz}_s{seed}")


# Time step of the batched cavities: dt = 0.05 h_min / (lid + sqrt(invEps)).
# At CFL 0.2 some of the 256 cavities (high lid speed, low viscosity) grow
# without bound within ~1000 steps - a property of the explicit scheme (the
# CPU restatement of the reference's solver diverges the same way) - so the
# batched workload runs at CFL 0.05.
BATCHED_CFL = 0.05


def batched_cavities(count: int = 256, seed: int = 0, n_lo: int = 8, n_hi: int = 48,
                     steps: int = 200) -> list:
    """The batched workload: `count` independent VMS cavities, each with its
    own seed; n ~ U{n_lo..n_hi} (6 n^3 tets), viscosity log-uniform in
    [1e-3, 1e-1] (rho = 1), lid speed uniform in [0.5, 2], CFL 0.05."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, count)
    nus = np.exp(rng.uniform(np.log(1e-3), np.log(1e-1), count))
    lids = rng.uniform(0.5, 2.0, count)
    return [cavity(int(n), seed=seed * 100003 + i, mu=float(nu), lid=float(lid), steps=steps, cfl=BATCHED_CFL)
            for i, (n, nu, lid) in enumerate(zip(ns, nus, lids))]


def _fmt_rows(prefix: str, first: np.ndarray, vals: np.ndarray | None = None, ints: np.ndarray | None = None) -> str:
    cols = [np.char.add(prefix, first.astype(str))]
    if vals is not None:
        for c in range(vals.shape[1]):
            cols.append(np.char.mod("%.17e", vals[:, c]))
    if ints is not None:
        cols.append(ints.astype(str))
    if not len(first):
        return ""
    out = cols[0]
    for c in cols[1:]:
        out = np.char.add(np.char.add(out, " "), c)
    return "\n".join(out.tolist()) + "\n"


def write_dat(p: Problem, path: str, output_prefix: str = "sol", log_file: str = "log.txt") -> None:
    """Write ``p`` as a reference-readable .dat keyword file."""
    with open(path, "w") as f:
        f.write("PROBLEM EXPLICITVMS\n")
        if p.solver == SUPG:
            f.write(f"NODEDOF {p.max_node_dofs} {p.glob_fixed}\n")
        else:
            f.write(f"NODEDOF {p.max_node_dofs}\n")
        f.write("TIMESTEP %.17e %d %d\n" % (p.time_step, p.total_steps, p.save_every))
        f.write("DUALSTEP %.17e %d\n" % (p.dual_step, p.tot_dual_steps))
        f.write("VMSPROPS " + " ".join("%.17e" % v for v in p.props) + "\n")
        f.write("EXOPTS " + " ".join(str(int(v)) for v in p.ex_opts) + "\n")
        f.write(f"OUTPUT {output_prefix}\nLOGFILE {log_file}\n")
        f.write("EXITCOND %.17e\n" % p.exit_condition)
        N = p.n_nodes
        f.write(_fmt_rows("NODE ", np.arange(1, N + 1), p.coords))
        et = "TET4" if p.elem_type == TET4 else "HEXA8"
        E = p.n_elems
        lines = np.char.add(f"ELEMENT {et} ", np.arange(1, E + 1).astype(str))
        lines = np.char.add(lines, " 1")
        for c in range(p.conn.shape[1]):
            lines = np.char.add(np.char.add(lines, " "), (p.conn[:, c].astype(np.int64) + 1).astype(str))
        f.write("\n".join(lines.tolist()) + "\n")
        f.write(_fmt_rows("NODEVEL ", p.vel_node + 1, p.vel_vals, p.vel_dir))
        f.write(_fmt_rows("NODEDIRBC ", p.dir_node + 1, p.dir_vals))
        f.write(_fmt_rows("NODEPRES ", p.pres_node + 1, p.pres_vals.reshape(-1, 1)))


# ---------------------------------------------------------------------------
# Poisson problems (femPoissonSolver::solve, femSolver.cpp:409-654)
# ---------------------------------------------------------------------------
POISSON_CLASSIC, POISSON_PPE, POISSON_DISTANCE = 0, 1, 2


@dataclass
class PoissonProblem:
    """The femModel fields femPoissonSolver::solve reads: mesh, per-element
    diffusivity (ELDIFF rows in element order), ELSOURCE rows, FACENEUMANN
    rows (face node lists in CSR form), NODEDIRBC rows (first value) and the
    PROBLEM type."""
    coords: np.ndarray
    conn: np.ndarray
    diffusivity: np.ndarray
    source_elem: np.ndarray
    source_value: np.ndarray
    neumann_off: np.ndarray
    neumann_nodes: np.ndarray
    neumann_value: np.ndarray
    dir_node: np.ndarray
    dir_value: np.ndarray
    problem: int = POISSON_CLASSIC
    name: str = "poisson"

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])


def poisson_box(n: int, elem_type: int = TET4, problem: int = POISSON_CLASSIC, seed: int = 0,
                jitter: float = 0.1, anisotropic: bool = True, sources: bool = True, neumann: bool = True,
                dirichlet: bool = True) -> PoissonProblem:
    """Unit cube, n^3 cells (6 Kuhn tets or one hexa8 each) with seeded
    interior jitter; seeded per-element diffusivity (each component in
    [0.5, 2] when anisotropic, else 1); an ELSOURCE row for every fourth
    element; FACENEUMANN rows on the x = 1 face (one per boundary face, its
    3 or 4 nodes); NODEDIRBC on the x = 0 face with a smooth value.  Without
    Dirichlet rows the system is singular (pure Neumann): the solver then
    works on the zero-sum part of the right-hand side."""
    rng = np.random.default_rng(seed + 7919)
    if elem_type == TET4:
        X, conn, _ = kuhn_cavity_mesh(n, seed, jitter)
    else:
        p = channel(n, n, n, seed=seed, jitter=jitter, steps=1)
        X = p.coords / np.array([4.0, 1.0, 1.0])  # the channel box scaled to the unit cube
        conn = p.conn
    E = conn.shape[0]
    diff = rng.uniform(0.5, 2.0, (E, 3)) if anisotropic else np.ones((E, 3))
    if sources:
        se = np.arange(0, E, 4, dtype=np.int32)
        sv = rng.uniform(-1.0, 1.0, se.size)
    else:
        se, sv = np.zeros(0, np.int32), np.zeros(0)
    tol = 1e-12
    on_x1 = X[:, 0] > 1.0 - tol
    if neumann:
        # boundary faces on x = 1: element faces whose nodes all lie there
        faces = []
        npe = conn.shape[1]
        face_sets = ([(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)] if npe == 4 else
                     [(0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)])
        for fs in face_sets:
            m = np.all(on_x1[conn[:, list(fs)]], axis=1)
            for e in np.nonzero(m)[0]:
                faces.append(conn[e, list(fs)])
        faces.sort(key=lambda f: tuple(sorted(f.tolist())))
        off = np.zeros(len(faces) + 1, np.int32)
        off[1:] = np.cumsum([len(f) for f in faces])
        nodes = np.concatenate(faces).astype(np.int32) if faces else np.zeros(0, np.int32)
        nval = rng.uniform(0.0, 1.0, len(faces))
    else:
        off, nodes, nval = np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)
    if dirichlet:
        dn = np.nonzero(X[:, 0] < tol)[0].astype(np.int32)
        dv = np.sin(np.pi * X[dn, 1]) * np.cos(np.pi * X[dn, 2])
    else:
        dn, dv = np.zeros(0, np.int32), np.zeros(0)
    return PoissonProblem(X, conn.astype(np.int32), diff, se, sv, off, nodes, nval, dn, dv, problem,
                          name=f"poisson{'tet' if elem_type == TET4 else 'hexa'}{n}_s{seed}")


def write_poisson_dat(pp: PoissonProblem, path: str) -> None:
    """Write ``pp`` as a reference-readable .dat keyword file (PROBLEM, NODE,
    ELEMENT, ELDIFF, ELSOURCE, FACENEUMANN, NODEDIRBC; femModel.cpp:
    3719-4213)."""
    kind = {POISSON_CLASSIC: "POISSON", POISSON_PPE: "PPE", POISSON_DISTANCE: "DISTANCE"}[pp.problem]
    with open(path, "w") as f:
        f.write(f"PROBLEM {kind}\n")
        N, E = pp.n_nodes, pp.n_elems
        f.write(_fmt_rows("NODE ", np.arange(1, N + 1), pp.coords))
        et = "TET4" if pp.conn.shape[1] == 4 else "HEXA8"
        lines = np.char.add(f"ELEMENT {et} ", np.arange(1, E + 1).astype(str))
        lines = np.char.add(lines, " 1")
        for c in range(pp.conn.shape[1]):
            lines = np.char.add(np.char.add(lines, " "), (pp.conn[:, c].astype(np.int64) + 1).astype(str))
        f.write("\n".join(lines.tolist()) + "\n")
        f.write(_fmt_rows("ELDIFF ", np.arange(1, E + 1), pp.diffusivity))
        f.write(_fmt_rows("ELSOURCE ", pp.source_elem + 1, pp.source_value.reshape(-1, 1)))
        for k in range(pp.neumann_value.size):
            nodes = pp.neumann_nodes[pp.neumann_off[k]:pp.neumann_off[k + 1]] + 1
            f.write("FACENEUMANN 1 " + " ".join(str(int(v)) for v in nodes) + " %.17e\n" % pp.neumann_value[k])
        f.write(_fmt_rows("NODEDIRBC ", pp.dir_node + 1, pp.dir_value.reshape(-1, 1)))
