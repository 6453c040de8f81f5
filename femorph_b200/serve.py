"""Continuous-batching request loop for VMS cavity solves on one GPU.

Requests (a mesh.Problem and a step count) arrive over time.  The server
keeps one batch whose device pools are sized once from an HBM budget
(fm_batch_create_empty); it builds each arriving problem's tile layout on a
host thread pool (fm_problem_prepare), admits prepared problems first come
first served whenever the pools have room (fm_batch_add returns FM_ERR_OOM
otherwise), advances every resident problem by up to `block` steps per round
in one launch pair per iteration (fm_batch_step_problems, ragged targets), and
retires finished problems (state read back, ranges freed) between rounds, so
requests that arrive while others run join the work on the device without
waiting for them to finish.  A problem's result does not depend on which other
problems share the batch (tiles never span problems; every launch is
deterministic).

Preemption (optional, `preempt_after` seconds): when the oldest prepared
request has waited that long for room, the resident solve with the most
steps left (among those that ran at least one round since admission) is
checkpointed to `spill_dir` (fm_problem_checkpoint), removed, and queued
behind the waiting requests; re-admitted, it is restored
(fm_problem_restore) and continues bit for bit.

The reference solves one model per process (femVMSExplicitFluidSolver::solve,
src/femVMSExplicitFluidSolver.cpp:842-1334); this loop has no counterpart
there.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import dataclasses
import os
import time

import numpy as np

from . import api, mesh

# Kuhn tet meshes have about 5.8 elements per node; the node pools are sized
# for 5 (small meshes have relatively more boundary nodes).
ELEMS_PER_NODE = 5.0


@dataclasses.dataclass
class Request:
    rid: int
    problem: mesh.Problem
    steps: int
    arrival: float                  # seconds after the start of the run
    admitted: float | None = None
    done: float | None = None
    result: tuple | None = None     # (u (N,3), p (N,)) after `steps` steps
    status: int = 0                 # FM_OK, or the device status that retired it early
    steps_done: int = 0
    preemptions: int = 0
    spill: str | None = None        # checkpoint of a preempted solve, until re-admitted
    blocked: float | None = None    # when it first found no room at the head of the queue

    @property
    def latency(self) -> float:
        return self.done - self.arrival

    @property
    def work(self) -> int:
        return self.problem.n_elems * self.steps_done


class Server:
    """One GPU, one pooled batch; see the module docstring."""

    def __init__(self, precision: int = api.FM_MIXED, hbm_budget: int = 16 << 30, max_problems: int = 512,
                 block: int = 50, device: int = 0, prepare_workers: int = 0, tuning: dict | None = None,
                 keep_results: bool = True, preempt_after: float | None = None, spill_dir: str | None = None):
        self.precision = precision
        self.block = block
        self.preempt_after = preempt_after
        self.spill_dir = spill_dir
        if preempt_after is not None and spill_dir is None:
            raise ValueError("preemption checkpoints to spill_dir")
        self.hbm_budget = hbm_budget
        self.keep_results = keep_results
        self.tuning = dict(tuning or {})
        # largest pools whose allocation fits the budget (bytes grow linearly
        # with the element capacity)
        probe = 10_000_000
        tk = {k: self.tuning[k] for k in ("tile_elems", "tile_nodes", "threads") if k in self.tuning}
        per = api.capacity_bytes(mesh.VMS, 4, max_problems, probe, int(probe / ELEMS_PER_NODE), precision, **tk)
        max_elems = int(probe * hbm_budget / per)
        max_nodes = int(max_elems / ELEMS_PER_NODE)
        self.pool = api.Pool(mesh.VMS, 4, max_problems=max_problems, max_elems=max_elems, max_nodes=max_nodes,
                             precision=precision, device=device, **self.tuning)
        self.capacity = dict(max_elems=max_elems, max_nodes=max_nodes, max_problems=max_problems)
        self.exec = cf.ThreadPoolExecutor(max_workers=prepare_workers or min(32, os.cpu_count() or 4))

    def _prepare(self, req: Request):
        g = api.GpuProblem(req.problem, self.precision)
        g.prepare(tile_elems=self.tuning.get("tile_elems", 0), tile_nodes=self.tuning.get("tile_nodes", 0),
                  threads=self.tuning.get("threads", 0))
        return g

    def run(self, requests: list[Request], clock=time.perf_counter) -> dict:
        """Serves `requests` (arrival times relative to the start); returns
        run statistics.  Blocks until every request is done."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        preparing: collections.deque = collections.deque()   # (req, future) in arrival order
        resident: list = []                  # [req, GpuProblem, remaining steps, steps since admission]
        rounds = 0
        preemptions = 0
        busy = 0.0
        peak_resident = 0
        t0 = clock()
        while pending or preparing or resident:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                preparing.append((r, self.exec.submit(self._prepare, r)))
            # admit prepared problems in arrival order while the pools have room
            while preparing and preparing[0][1].done():
                r, fut = preparing[0]
                g = fut.result()
                if not self.pool.add(g):
                    if not resident:
                        raise RuntimeError(f"request {r.rid} ({r.problem.n_elems} elements) does not fit the "
                                           f"server's pools {self.capacity}")
                    if r.blocked is None:
                        r.blocked = now
                    break
                preparing.popleft()
                r.blocked = None
                if r.spill is not None:
                    g.restore(r.spill)
                    os.remove(r.spill)
                    r.spill = None
                if r.admitted is None:
                    r.admitted = clock() - t0
                resident.append([r, g, r.steps - r.steps_done, 0])
            if (self.preempt_after is not None and preparing and preparing[0][0].blocked is not None
                    and now - preparing[0][0].blocked >= self.preempt_after):
                movable = [item for item in resident if item[3] >= self.block]
                if movable:
                    victim = max(movable, key=lambda item: item[2] * item[0].problem.n_elems)
                    v, g, _, _ = victim
                    v.spill = os.path.join(self.spill_dir, f"request{v.rid}.fmck")
                    g.checkpoint(v.spill)
                    self.pool.remove(g)
                    resident.remove(victim)
                    v.preemptions += 1
                    preemptions += 1
                    fut: cf.Future = cf.Future()
                    fut.set_result(g)
                    preparing.append((v, fut))
                    continue
            if not resident:
                # idle: wait for the next arrival or preparation
                if preparing:
                    cf.wait([preparing[0][1]], timeout=0.05)
                elif pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                continue
            peak_resident = max(peak_resident, len(resident))
            steps = [min(self.block, item[2]) for item in resident]
            ts = clock()
            self.pool.step([item[1] for item in resident], steps)
            failed = self.pool.wait()   # True when some problem reported a device error
            busy += clock() - ts
            rounds += 1
            still = []
            for item, k in zip(resident, steps):
                item[2] -= k
                item[3] += k
                r, g, rem, _ = item
                r.steps_done += k
                status = g.status() if failed else api.FM_OK
                if rem > 0 and status == api.FM_OK:
                    still.append(item)
                    continue
                # finished, or retired early: diverged (NaN/Inf) or a BC table
                # lookup failed; the other problems are unaffected
                r.status = status
                if self.keep_results:
                    u, p, _, _ = g.state(elements=False)
                    r.result = (u, p)
                self.pool.remove(g)
                g.close()
                r.done = clock() - t0
            resident = still
        total = clock() - t0
        lat = np.array([r.latency for r in requests])
        work = sum(r.work for r in requests)
        first = min(r.arrival for r in requests)
        last = max(r.done for r in requests)
        return {"requests": len(requests), "rounds": rounds, "wall_s": total, "gpu_busy_s": busy,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_latency_s": float(lat.mean()), "element_steps": int(work),
                "element_steps_per_s": work / (last - first), "peak_resident": peak_resident,
                "failed": sum(1 for r in requests if r.status != 0), "preemptions": preemptions}

    def close(self):
        self.exec.shutdown(wait=True)
        self.pool.close()


def draw_requests(count: int, rate: float, seed: int = 0, n_range=(12, 64), steps_range=(100, 2000),
                  problems: list | None = None) -> list[Request]:
    """Served-stream requests: Poisson arrivals at `rate` per second; per
    request n ~ U{n_range}, steps ~ U{steps_range}, viscosity log-uniform in
    [1e-3, 1e-1] (rho = 1), lid speed ~ U[0.5, 2], its own mesh/noise seed.
    `problems` reuses already generated meshes (same draws) with new arrival
    times."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_range[0], n_range[1] + 1, count)
    steps = rng.integers(steps_range[0], steps_range[1] + 1, count)
    nus = np.exp(rng.uniform(np.log(1e-3), np.log(1e-1), count))
    lids = rng.uniform(0.5, 2.0, count)
    gaps = np.random.default_rng(seed + 7919).exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps) - gaps[0]
    out = []
    for i in range(count):
        p = problems[i] if problems is not None else make_problem(int(ns[i]), float(nus[i]), float(lids[i]),
                                                                 seed * 100003 + i)
        out.append(Request(rid=i, problem=p, steps=int(steps[i]), arrival=float(arrivals[i])))
    return out


def request_params(count: int, seed: int = 0, n_range=(12, 64)):
    """(n, nu, lid, mesh seed) of each request, as draw_requests draws them."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_range[0], n_range[1] + 1, count)
    rng.integers(100, 2001, count)
    nus = np.exp(rng.uniform(np.log(1e-3), np.log(1e-1), count))
    lids = rng.uniform(0.5, 2.0, count)
    return [(int(ns[i]), float(nus[i]), float(lids[i]), seed * 100003 + i) for i in range(count)]


# Served requests run up to 2000 steps; with dt = 0.2 h_min / (lid +
# sqrt(invEps)) the reference algorithm itself (the oracle) blows up within
# about 600 steps on these cavities, so the stream uses CFL 0.05, with which
# 2000 steps stay bounded by the lid speed.
SERVE_CFL = 0.05


def make_problem(n: int, nu: float, lid: float, seed: int) -> mesh.Problem:
    return mesh.cavity(n, seed=seed, mu=nu, lid=lid, steps=2001, cfl=SERVE_CFL)
