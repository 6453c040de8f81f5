"""Benchmark: VMS explicit step on the 96^3 Kuhn-tet lid-driven cavity.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 96] [--precision fp64|mixed|both]

Workload (one GPU): unit cube, 96^3 cells x 6 Kuhn tets = 5,308,416 tet4 and
912,673 nodes, interior jitter +-0.1h, lid u=(1,0,0), no-slip walls,
rho=1, mu=0.01, invEps=400, c1=4, c2=2, dt = 0.2 h_min/(1+sqrt(invEps)),
seeded +-1e-3 initial noise.  A "step" is one time step (one dual iteration)
of femVMSExplicitFluidSolver over the whole mesh.  Inputs (5.3 M elements x
96 B of subscales, ~0.5 GB) exceed the 126 MB L2, so no L2 flush is needed
between steps.  With --gpus N each rank solves its own cavity (seed = rank):
weak scaling, no data-path collective; value = element-steps/s summed over
ranks with the time taken as the max over ranks.  --config partitioned
splits ONE cavity over the N ranks instead (strong scaling, one all-reduce
of the shared nodes' partial sums per dual iteration).

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic_per_element.json")


def measured_traffic(kernel: str, precision: str, E: int):
    """DRAM bytes (read + write) of one launch of `kernel`, from the ncu
    capture summarised in profiles/: bytes per element measured on a smaller
    mesh of the same family, scaled by the element count (traffic grows in
    proportion).  None when no capture is recorded."""
    try:
        with open(TRAFFIC_FILE) as f:
            d = json.load(f)
        return d[kernel][precision]["bytes_per_element"] * E
    except Exception:
        return None


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(E: int, N: int, precision: str, config: str = "cavity") -> int:
    """Compulsory HBM bytes of one step.  VMS: per element connectivity (4 x
    int32) and the 12 Gauss-point subscales read and written; per node
    coordinates, the 4-dof state read and written and the lumped mass.  SUPG
    (Euler, no history): per element connectivity (npe x int32); per node
    coordinates, velocity read and written and the lumped mass.  Derived
    geometry is not counted (it can be formed from the coordinates); the
    FP64 hexa8 kernel's stored Gauss-point geometry is reported beside it
    (stored_geometry_bytes)."""
    if config == "cavity":
        sub = 48 if precision == "mixed" else 96
        return E * (16 + 2 * sub) + N * (24 + 32 + 32 + 8)
    npe = 8 if config == "channel" else 4
    return E * 4 * npe + N * (24 + 24 + 24 + 8)


def stored_geometry_bytes(E: int, precision: str, config: str) -> int:
    """Bytes of stored Gauss-point geometry one FP64 hexa8 step reads (8
    points x 10 FP64 values an element); 0 for the other kernels."""
    return E * 8 * 10 * 8 if config == "channel" and precision != "mixed" else 0


# FP64 operations of one SUPG element-step (matrix-free K u over the Gauss
# points, counting an FMA as two), from the ncu FP64 instruction counts of
# the tile kernels (profiles/supg_tile_kernel_*.md); the hexa8 count is that
# of the kernel reading the stored Gauss-point geometry.
SUPG_FLOPS = {"channel": 6419, "supg": 1676}

CONFIG_DEFAULT_N = {"cavity": 96, "supg": 96, "channel": 64, "io": 96}


def make_problem(args, seed: int, n: int | None = None):
    """The configured single-GPU workload: 'cavity' VMS Kuhn cavity n^3 x 6
    tets; 'supg' the same mesh with the SUPG solver (Euler, K1-K4, no B-bar);
    'channel' the hexa8 channel 4n x n x n (256 x 64 x 64 at n = 64), SUPG."""
    from femorph_b200 import mesh
    n = n or args.n
    if args.config == "supg":
        # CFL 0.2 (dt = 0.2 h_min / lid) lets the explicit SUPG cavity grow
        # without bound within a few dozen steps at 48^3 and above; 0.05 stays
        # bounded by the lid speed for 300+ steps at 96^3
        return mesh.cavity(n, seed=seed, steps=200, solver=mesh.SUPG, cfl=0.05)
    if args.config == "channel":
        return mesh.channel(4 * n, n, n, seed=seed, steps=500)
    return mesh.cavity(n, seed=seed, steps=200)


def run_ours(args, rank, world, local_rank, dist):
    from femorph_b200 import api, mesh

    prec = api.FM_MIXED if args.precision == "mixed" else api.FM_FP64
    p = make_problem(args, seed=rank)
    E, N = p.n_elems, p.n_nodes
    g = api.GpuProblem(p, prec)
    tune = dict(tile_elems=args.tile_elems, tile_nodes=args.tile_nodes, threads=args.threads,
                ctas_per_sm=args.ctas_per_sm)
    b = api.Batch([g], device=local_rank, **tune)
    b.step(args.warmup)
    b.sync()
    if dist:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        b.step(args.steps)
        b.sync()
    ms, launches = b.last_timing()
    if dist:
        import torch
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # per-kernel profile (separate, shorter run)
    kprof, klaunch = b.profile(min(args.steps, 50))
    b.sync()
    lay = b.layout()
    state = g.state(elements=False)[:2]
    b.close()
    g.close()
    res = dict(E=E, N=N, ms=ms, launches=launches, clocks=clk.summary(), kprof=kprof, klaunch=klaunch, layout=lay,
               state=state, steps_total=args.warmup + args.steps + min(args.steps, 50), p=p)
    # end to end through the C ABI: the whole solve of the configured
    # problem (its own step count) from host buffers to the state read back
    if rank == 0:
        e2e_steps = p.steps
        t0 = time.perf_counter()
        g2 = api.GpuProblem(p, prec)
        b2 = api.Batch([g2], device=local_rank, **tune)
        b2.step(e2e_steps)
        b2.sync()
        u, pr, _, _ = g2.state(elements=False)
        t1 = time.perf_counter()
        b2.close()
        g2.close()
        res["e2e_s"] = t1 - t0
        res["e2e_steps"] = e2e_steps
        res["h2d"] = p.coords.nbytes + p.conn.nbytes + p.init_state.nbytes
        res["d2h"] = u.nbytes + pr.nbytes
    return res


def accuracy_run(args, local_rank, steps: int):
    """Mixed form against the FP64 form on the GPU after `steps` steps of
    the configured workload (fresh solves of the same problem)."""
    from femorph_b200 import api
    p = make_problem(args, seed=0)
    out = {}
    for pn, prec in (("fp64", api.FM_FP64), ("mixed", api.FM_MIXED)):
        g = api.GpuProblem(p, prec)
        b = api.Batch([g], device=local_rank)
        b.step(steps)
        b.sync()
        out[pn] = g.state(elements=False)[:2]
        b.close()
        g.close()
    (um, pm), (ud, pd) = out["mixed"], out["fp64"]
    return {"u": float(np.linalg.norm(um - ud) / np.linalg.norm(ud)),
            "p": float(np.linalg.norm(pm - pd) / max(np.linalg.norm(pd), 1e-300)),
            "after_steps": steps,
            "reference": "the FP64 GPU path (itself within 1e-10 of the oracle after 200 steps of this "
                         "workload, tests/test_gpu_fullsize.py)"}


def batched_problems(count: int = 256, seed: int = 0):
    """Batched workload (femorph_b200.mesh.batched_cavities): `count`
    independent cavities, n ~ U{8..48}, viscosity log-uniform in
    [1e-3, 1e-1], lid speed uniform in [0.5, 2], CFL 0.05."""
    from femorph_b200 import mesh
    return mesh.batched_cavities(count, seed=seed)


def run_batched(args, rank, world, local_rank, dist):
    """Config 4 on each rank: the rank's share of the problems in one batch
    (one launch pair per step for all of them), 50-step CUDA graphs, launch
    shape from the autotuner.  Also runs the FP64 form on the same problems
    and reports the mixed-vs-FP64 relative L2 after the timed steps."""
    from femorph_b200 import api, shard
    probs = batched_problems(args.batch_count, seed=args.seed)
    costs = [p.n_elems for p in probs]
    owned = shard.mine(costs, world, rank)
    probs = [probs[i] for i in owned]
    E = sum(p.n_elems for p in probs)
    res = {}
    states = {}
    for prec_name, prec in (("mixed", api.FM_MIXED), ("fp64", api.FM_FP64)):
        gs = [api.GpuProblem(p, prec) for p in probs]
        cache = os.path.join(ROOT, "femorph_b200", "autotune_cache.txt")
        tune = api.autotune(gs[:16], device=local_rank, steps=5, cache_path=cache)
        b = api.Batch(gs, device=local_rank, graph_steps=50, **tune)
        b.step(args.warmup)
        b.sync()
        if dist:
            dist.barrier()
        with ClockSampler(local_rank) as clk:
            b.step(args.steps)
            b.sync()
        ms, launches = b.last_timing()
        ms = shard.reduce_max(ms, dist, f"cuda:{local_rank}")
        kprof, klaunch = b.profile(min(args.steps, 50))
        states[prec_name] = [g.state()[:2] for g in gs]
        res[prec_name] = dict(ms=ms, launches=launches, clocks=clk.summary(), kprof=kprof, klaunch=klaunch,
                              tune=tune, layout=b.layout())
        b.close()
        for g in gs:
            g.close()
    err_u = max(np.linalg.norm(a[0] - b_[0]) / max(np.linalg.norm(b_[0]), 1e-300)
                for a, b_ in zip(states["mixed"], states["fp64"]))
    err_p = max(np.linalg.norm(a[1] - b_[1]) / max(np.linalg.norm(b_[1]), 1e-300)
                for a, b_ in zip(states["mixed"], states["fp64"]))
    res["E"] = E
    res["E_total"] = shard.reduce_sum(E, dist, f"cuda:{local_rank}")
    res["err"] = (err_u, err_p)
    res["N"] = sum(p.n_nodes for p in probs)
    return res


def run_poisson(args, rank, world, local_rank, dist):
    """The Poisson solver (femPoissonSolver::solve) on an n^3 Kuhn-tet cube:
    each timed step is one whole preconditioned-CG solve from x = 0 to a
    relative residual of 1e-10 on the device (host assembly and upload are
    outside the timed region, which is what e2e adds)."""
    from femorph_b200 import api, mesh

    n = args.n or 96
    p = mesh.poisson_box(n, mesh.TET4, seed=rank)
    s = api.GpuPoisson(p, device=local_rank)
    rows, nnz = s.info()
    for _ in range(max(1, args.warmup)):
        s.solve(1e-10, 100000)
    if dist:
        dist.barrier()
    iters, dev_ms = 0, 0.0
    solves = max(1, args.steps)
    with ClockSampler(local_rank) as clk:
        for _ in range(solves):
            it, rr, ms = s.solve(1e-10, 100000)
            iters += it
            dev_ms += ms
    s.close()
    if dist:
        import torch
        t = torch.tensor([dev_ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    res = dict(n=n, N=p.n_nodes, E=p.n_elems, nnz=nnz, iters=iters, solves=solves, ms=dev_ms, clocks=clk.summary(),
               rr=rr)
    if rank == 0:
        # end to end through the C ABI: host assembly + upload + solve + read-back
        t0 = time.perf_counter()
        s2 = api.GpuPoisson(p, device=local_rank)
        it2, _, _ = s2.solve(1e-10, 100000)
        x, _ = s2.solution()
        t1 = time.perf_counter()
        s2.close()
        res["e2e_s"], res["e2e_iters"] = t1 - t0, it2
        res["h2d"] = p.coords.nbytes + p.conn.nbytes + p.diffusivity.nbytes
        res["d2h"] = x.nbytes
        if not args.no_cpu:
            res["cpu"] = poisson_cpu_baseline(p)
    return res


def poisson_cpu_baseline(p, iters: int = 200):
    """The same Jacobi-preconditioned CG on the host (scipy sparse matrix of
    the oracle's assembly of the reference's system), a bounded number of
    iterations."""
    import scipy.sparse as sp
    from oracle import oracle_b

    K, b, _ = oracle_b.poisson_system(p)
    dinv = 1.0 / K.diagonal()
    x = np.zeros_like(b)
    r = b.copy()
    z = dinv * r
    q = z.copy()
    rz = r @ z
    t0 = time.perf_counter()
    for _ in range(iters):
        w = K @ q
        a = rz / (q @ w)
        x += a * q
        r -= a * w
        z = dinv * r
        rz2 = r @ z
        q = z + (rz2 / rz) * q
        rz = rz2
    dt = time.perf_counter() - t0
    return {"value": p.n_nodes * iters / dt, "unit": "DOF-iterations/s", "cores": 1, "kind": "port",
            "sample": f"{iters} Jacobi-PCG iterations on the oracle's assembly of the same system (scipy CSR, "
                      f"numpy vectors, one host thread)"}


def poisson_line(args, world, r):
    peak, peak_kind = hbm_peak()
    N, nnz = r["N"], r["nnz"]
    # compulsory bytes of one CG iteration: the matrix (value + column), row
    # offsets and the vectors each kernel reads or writes once (p, q in the
    # product; x, p, r, q, z, D^-1 in the update; z, p in the direction)
    ab = 12 * nnz + 4 * (N + 1) + 8 * N * 13
    ms_it = r["ms"] / max(1, r["iters"])
    achieved = ab / (ms_it * 1e-3) / 1e9
    value = world * N * r["iters"] / (r["ms"] / 1e3)
    line = {"metric": "Poisson CG DOF-iterations/s (Jacobi-PCG to 1e-10, n^3 Kuhn-tet cube)", "value": value,
            "unit": "DOF-iterations/s", "n_gpus": world, "steps": r["solves"], "warmup": args.warmup,
            "ms_per_step": r["ms"] / r["solves"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"femPoissonSolver on the {r['n']}^3 Kuhn-tet cube ({r['E']} tets, {N} nodes, "
                                   f"{nnz} matrix entries), anisotropic diffusivity, sources, Neumann and Dirichlet "
                                   f"faces; a step is one whole CG solve ({r['iters'] // r['solves']} iterations)",
                       "l2": "matrix and vectors larger than L2 (no flush)",
                       "parallelism": f"{world} independent solve(s), one per GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind, "kernel": "CG iteration (3 kernels)",
                         "algorithmic_bytes_per_iteration": ab, "avg_iteration_ms": ms_it},
            "gpu_launches": 3 * r["iters"] + 3 * r["solves"], "clocks": r["clocks"]}
    if "e2e_s" in r:
        line["e2e"] = {"value": N * r["e2e_iters"] / r["e2e_s"], "unit": "DOF-iterations/s",
                       "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                       "note": "one whole solve through the C ABI: host assembly + upload + CG + read-back, wall clock"}
    if "cpu" in r:
        line["cpu_baseline"] = r["cpu"]
    return line


def batched_line(args, world, rb):
    peak, peak_kind = hbm_peak()
    out = {}
    for pn in ("mixed", "fp64"):
        r = rb[pn]
        kl = max(1, r["klaunch"])
        tile_ms = r["kprof"]["tile"] / kl
        ab = algorithmic_bytes(rb["E"], rb["N"], pn)
        out[pn] = {"value": rb["E_total"] * args.steps / (r["ms"] / 1e3), "ms_per_step": r["ms"] / args.steps,
                   "tuning": r["tune"], "gpu_launches": r["launches"], "clocks": r["clocks"],
                   "roofline": {"bound": "hbm", "achieved": ab / (tile_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                "frac": ab / (tile_ms * 1e-3) / 1e9 / peak, "traffic": None,
                                "peak_source": peak_kind, "kernel": "vms_tile_kernel",
                                "algorithmic_bytes_per_launch": ab, "avg_launch_ms": tile_ms}}
    from femorph_b200 import mesh
    m = out["fp64"]
    return {"metric": "VMS element-steps/s, batched cavities (FP64; mixed beside)", "value": m["value"],
            "unit": "element-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.batch_count} independent VMS cavities per GPU job, n~U{{8..48}}, "
                                   f"nu log-U[1e-3,1e-1], lid U[0.5,2], CFL {mesh.BATCHED_CFL}, one launch pair per step for all, "
                                   f"50-step CUDA graphs, autotuned tiles", "elements": rb["E_total"],
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"problems sharded over {world} GPU(s) by LPT on element count"},
            "roofline": m["roofline"], "gpu_launches": m["gpu_launches"], "clocks": m["clocks"],
            "tuning": m["tuning"], "mixed": dict(out["mixed"], dtype="f32+f64"),
            "mixed_over_fp64": out["mixed"]["value"] / m["value"],
            "mixed_vs_fp64_rel_l2": {"u_max_over_problems": rb["err"][0], "p_max_over_problems": rb["err"][1],
                                     "after_steps": args.warmup + args.steps + min(args.steps, 50)}}


def _gen_request_problem(args):
    from femorph_b200 import serve
    return serve.make_problem(*args)


def run_serve(args, local_rank):
    """Config 5: Poisson stream of cavity solves (n ~ U{12..64}, steps ~
    U{100..2000}, nu log-U[1e-3,1e-1], lid U[0.5,2], per-request seed) served
    by femorph_b200.serve.Server under a stated HBM budget, at each arrival
    rate, for each precision.  The meshes are generated before the timed runs
    (client side, spawned processes) and reused across rates."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from femorph_b200 import api, serve
    params = serve.request_params(args.requests, seed=args.seed)
    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        problems = list(ex.map(_gen_request_problem, params))
    rates = [float(x) for x in args.rates.split(",")]
    budget = int(args.budget_gb * (1 << 30))
    precs = [("mixed", api.FM_MIXED), ("fp64", api.FM_FP64)]
    if args.precision != "both":
        precs = [x for x in precs if x[0] == args.precision]
    out = {}
    for pn, prec in precs:
        rows = []
        for rate in rates:
            reqs = serve.draw_requests(args.requests, rate, seed=args.seed, problems=problems)
            srv = serve.Server(precision=prec, hbm_budget=budget, max_problems=256, block=50, device=local_rank,
                               keep_results=False)
            with ClockSampler(local_rank) as clk:
                st = srv.run(reqs)
            srv.close()
            mean_work = sum(r.problem.n_elems * r.steps for r in reqs) / len(reqs)
            st.update({"rate_req_per_s": rate, "offered_element_steps_per_s": rate * mean_work,
                       "clocks": clk.summary(), "capacity": srv.capacity})
            rows.append(st)
        out[pn] = rows
    return out


def serve_line(args, res):
    head = "mixed" if "mixed" in res else "fp64"
    rows = res[head]
    top = rows[-1]
    return {"metric": "served VMS cavity stream: aggregate element-steps/s with p50/p99 latency",
            "value": top["element_steps_per_s"], "unit": "element-steps/s", "n_gpus": 1, "steps": None,
            "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if head == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"{args.requests} cavity requests per rate, Poisson arrivals, n~U{{12..64}}, "
                                   f"steps~U{{100..2000}}, nu log-U[1e-3,1e-1], lid U[0.5,2], dt from CFL 0.05 "
                                   f"on lid+sqrt(invEps); continuous batching, "
                                   f"50-step rounds, HBM budget {args.budget_gb} GiB",
                       "rates_req_per_s": args.rates, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": "one GPU, one pooled batch"},
            "p50_latency_s": top["p50_latency_s"], "p99_latency_s": top["p99_latency_s"],
            "serving": res, "clocks": top["clocks"]}


def run_partitioned(args, rank, world, local_rank, dist, prec_name):
    """One 96^3 VMS cavity split into `world` parts (Morton bands), one part
    per GPU; each dual iteration ends with one all-reduce of the shared
    nodes' partial sums (femorph_b200.partition).  Strong scaling: the
    whole mesh's element-steps per second, time = max over ranks of the
    CUDA-event time of K steps on each part's stream."""
    import torch
    from femorph_b200 import api
    from femorph_b200.partition import PartitionedSolve
    a2 = argparse.Namespace(**vars(args))
    a2.config = "cavity"
    p = make_problem(a2, seed=0)
    prec = api.FM_MIXED if prec_name == "mixed" else api.FM_FP64
    ps = PartitionedSolve(p, prec, device=local_rank, tile_elems=args.tile_elems, tile_nodes=args.tile_nodes,
                          threads=args.threads, graph_steps=args.graph_steps)
    ps.step(args.warmup)
    ps.prepare_graph()   # recorded before the timed region (no-op without --graph-steps)
    ps.sync()
    if dist:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        t0.record(ps.stream)
        ps.step(args.steps)
        t1.record(ps.stream)
        ps.sync()
    ms = t0.elapsed_time(t1)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    res = dict(E=p.n_elems, N=p.n_nodes, part_elems=ps.part.n_elems, part_nodes=ps.part.n_nodes,
               x_total=ps.part.x_total, count=ps.count, ms=ms, clocks=clk.summary(),
               shared_local=int((ps.part.xidx >= 0).sum()))
    ps.close()
    return res


def partitioned_line(args, world, runs):
    head = "mixed" if "mixed" in runs else "fp64"
    r = runs[head]
    val = r["E"] * args.steps / (r["ms"] / 1e3)
    line = {"metric": "VMS element-steps/s, one 96^3 Kuhn-tet cavity partitioned over the GPUs",
            "value": val, "unit": "element-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64" if head == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"VMS tet4 lid-driven cavity {args.n}^3 cells x 6 Kuhn tets ({r['E']} tets, "
                                   f"{r['N']} nodes), split into {world} Morton-band part(s), {head} form",
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"one mesh, {world} part(s), one part per GPU; one all-reduce of "
                                      f"{r['count']} doubles (the shared nodes' partial sums) per dual iteration",
                       "exchange_nodes": r["x_total"], "part_elements_rank0": r["part_elems"],
                       "graph_steps": args.graph_steps},
            "gpu_launches": 3 * args.steps, "clocks": r["clocks"]}
    if "fp64" in runs and head != "fp64":
        f = runs["fp64"]
        line["fp64"] = {"value": f["E"] * args.steps / (f["ms"] / 1e3), "ms_per_step": f["ms"] / args.steps}
    return line


def host_cpu() -> dict:
    """Host CPU model and core count (the CPU baselines use one core)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "cores_total": os.cpu_count(), "cores_used": 1}


def cpu_sample_n(args) -> int:
    """Mesh size of the bounded CPU sample: the full mesh for the tet
    configs (a few seconds per step), a 64 x 16 x 16 channel for the hexa
    one (the full 1 M hexa take minutes per step on one core)."""
    return 16 if args.config == "channel" else args.n


def cpu_baseline(args, steps: int = 2):
    """Oracle B (plain-C restatement, element loops on all host threads,
    nodal sums in the reference's element order) on `steps` steps of the
    workload (or of the bounded sample of cpu_sample_n)."""
    from oracle import oracle_b
    n = cpu_sample_n(args)
    p = make_problem(args, seed=0, n=n)
    o = oracle_b.OracleSolve(p)
    threads = oracle_b.get_threads()
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    solver = "femVMSExplicitFluidSolver" if args.config == "cavity" else "femSUPGExplicitFluidSolver"
    host = dict(host_cpu(), cores_used=threads)
    return {"value": p.n_elems * steps / dt, "unit": "element-steps/s", "cores": threads, "kind": "port",
            "host": host,
            "sample": f"{steps} time step(s) of {workload_name(args, n)} ({p.n_elems} elements) with the "
                      f"C restatement of {solver} on {threads} host threads, setup excluded"}


def io_file(args):
    """The cavity workload's input file, written once into a temporary
    directory (mesh.write_dat: the reference's .dat keywords)."""
    from femorph_b200 import mesh
    d = tempfile.mkdtemp(prefix="fm_io_")
    path = os.path.join(d, f"cavity{args.n}.dat")
    mesh.write_dat(mesh.cavity(args.n, seed=args.seed, steps=2), path)
    return d, path


def run_io(args):
    """--config io: the .dat reader (fm_problem_read_dat: the keywords of
    femModel::ReadFromFEMTextFile, femModel.cpp:3719-4213, parsed in blocks on
    the host threads) on the cavity's input file; a step is one whole read
    from the file into a problem (parse, checks, BC resolution, lumped mass).
    Each writer (legacy ASCII VTK, legacy binary VTK, VTU) is then timed on
    the problem: with a device placed in a batch (the state's read-back
    inside the timed write), without one on its initial state."""
    import ctypes as C
    import shutil
    import types

    from femorph_b200 import api
    d, path = io_file(args)
    size = os.path.getsize(path)
    L = api.lib()
    steps, warm = max(1, min(args.steps, 10)), max(1, min(args.warmup, 3))
    times, h = [], None
    try:
        for k in range(warm + steps):
            if h is not None:
                L.fm_problem_destroy(h)
            h = C.c_void_p()
            t0 = time.perf_counter()
            api.check(L.fm_problem_read_dat(path.encode(), 0, api.FM_FP64, C.byref(h)))
            if k >= warm:
                times.append(time.perf_counter() - t0)
        try:
            import torch
            has_gpu = torch.cuda.is_available()
        except Exception:
            has_gpu = False
        # with a device the problem's state is read back from the batch;
        # without one the writers export the initial state of the problem
        b = api.Batch([types.SimpleNamespace(h=h)]) if has_gpu else None
        writers = {"state": "device (read back inside the timed write)" if b else "initial (no device)"}
        for name, fn in (("vtk_ascii", L.fm_problem_write_vtk), ("vtk_binary", L.fm_problem_write_vtk_binary),
                         ("vtu", L.fm_problem_write_vtu)):
            out = os.path.join(d, "out." + ("vtu" if name == "vtu" else "vtk"))
            ws = []
            for k in range(2):
                t0 = time.perf_counter()
                api.check(fn(h, out.encode()))
                ws.append(time.perf_counter() - t0)
            osz = os.path.getsize(out)
            writers[name] = {"bytes": osz, "s": min(ws), "MB_per_s": osz / min(ws) / 1e6}
            os.remove(out)
        if b is not None:
            b.close()
    finally:
        if h is not None:
            L.fm_problem_destroy(h)
        shutil.rmtree(d, ignore_errors=True)
    return {"size": size, "times": times, "warm": warm, "writers": writers}


def io_reference(args, path):
    """The reference's own reader (femModel::ReadFromFEMTextFile, compiled
    here as oracle/_ref/fm_refdrv, mode parse) on the same file: seconds."""
    from oracle import ref
    tf = path + ".timing"
    r = subprocess.run([ref.REFDRV, path, "parse", "--timing", tf], capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    with open(tf) as f:
        for line in f:
            if line.startswith("# parsed"):
                return float(line.split()[2])
    raise RuntimeError("no parse time recorded")


def io_config(args, size):
    return {"workload": f"reader of the {args.n}^3 Kuhn-tet cavity .dat ({size / 1e6:.1f} MB, "
                        f"{6 * args.n ** 3} TET4 elements, {(args.n + 1) ** 3} nodes)",
            "host_threads": os.cpu_count(), "l2": "host-only path"}


def io_line(args, world, r):
    t = np.array(r["times"])
    sec = float(np.median(t))
    val = r["size"] / sec / 1e6
    line = {"metric": ".dat read throughput (file to problem, C ABI)", "value": val, "unit": "MB/s",
            "n_gpus": world, "steps": len(t), "warmup": r["warm"], "ms_per_step": 1e3 * sec,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": io_config(args, r["size"]), "read_s": {"median": sec, "min": float(t.min())},
            "writers": r["writers"], "host": host_cpu() | {"cores_used": os.cpu_count()}}
    if not args.no_cpu:
        from oracle import ref
        if ref.available():
            d, path = io_file(args)
            try:
                rs = io_reference(args, path)
            finally:
                import shutil
                shutil.rmtree(d, ignore_errors=True)
            line["cpu_baseline"] = {"value": r["size"] / rs / 1e6, "unit": "MB/s", "cores": 1, "kind": "reference",
                                    "sample": "one read of the same file by femModel::ReadFromFEMTextFile "
                                              "(reference sources, single-threaded)"}
    return line


def run_reference(args):
    """The reference's own CPU solver (oracle A = the reference sources compiled
    in this repository) on a bounded sample of the workload: the full mesh,
    W warm-up + K timed time steps, parse and setup excluded."""
    from oracle import ref
    from femorph_b200 import mesh
    if args.config == "poisson":
        return {"impl": "reference", "unavailable": "the reference solves the Poisson system only through Trilinos "
                                                    "(src/femSolver.cpp:590-600), which is not in this image"}
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/fm_refdrv was not built (reference sources absent)"}
    if args.config == "io":
        d, path = io_file(args)
        try:
            size = os.path.getsize(path)
            rs = [io_reference(args, path) for _ in range(max(1, min(args.steps, 3)))]
        finally:
            import shutil
            shutil.rmtree(d, ignore_errors=True)
        sec = float(np.median(rs))
        val = size / sec / 1e6
        return {"impl": "reference", "metric": ".dat read throughput (file to problem, C ABI)", "value": val,
                "unit": "MB/s", "n_gpus": args.gpus, "steps": len(rs), "warmup": 0, "ms_per_step": 1e3 * sec,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": io_config(args, size),
                "cpu_baseline": {"value": val, "unit": "MB/s", "cores": 1, "kind": "reference",
                                 "sample": f"{len(rs)} whole reads by femModel::ReadFromFEMTextFile "
                                           "(reference sources, single-threaded)"},
                "e2e": {"value": val, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    n = cpu_sample_n(args)
    steps = max(1, min(args.steps, args.ref_steps))
    warm = max(1, min(args.warmup, 1))
    p = make_problem(args, seed=0, n=n)
    p.total_steps = steps + warm + 1
    p.save_every = 10 ** 9
    wd = tempfile.mkdtemp(prefix="fm_refbench_")
    out = ref.run(p, workdir=wd, timing=True, timeout=3600)
    st = out["timing"]["stamps"]
    # stamps: initial call (t=0) then one per step (after its element loops)
    t = st[:, 0]
    per = np.diff(t[1:])[warm - 1:] if len(t) > 2 else np.array([np.nan])
    per = per[-steps:]
    sec = float(np.sum(per))
    val = p.n_elems * len(per) / sec
    cores = 1
    return {"impl": "reference", "metric": METRIC[args.config], "value": val, "unit": "element-steps/s",
            "n_gpus": args.gpus,
            "steps": len(per), "warmup": warm, "ms_per_step": 1e3 * sec / len(per), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": val, "unit": "element-steps/s", "cores": cores, "kind": "reference",
                             "host": host_cpu(),
                             "sample": f"{len(per)} timed steps after {warm} warm-up of {workload_name(args, n)} "
                                       f"({p.n_elems} elements) through "
                                       f"{'femVMSExplicitFluidSolver' if args.config == 'cavity' else 'femSUPGExplicitFluidSolver'}"
                                       f"::solve (reference sources, g++ -O2), parse/setup excluded; the reference "
                                       f"is single-threaded"},
            "e2e": {"value": val, "unit": "element-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


METRIC = {"cavity": "VMS element-steps/s (explicit step, 96^3 Kuhn-tet cavity)",
          "supg": "SUPG tet4 element-steps/s (explicit step, 96^3 Kuhn-tet cavity)",
          "channel": "SUPG hexa8 element-steps/s (explicit step, 256x64x64 channel)"}


def workload_name(args, n):
    if args.config == "channel":
        return f"the hexa8 channel {4 * n}x{n}x{n}"
    return f"the {n}^3 Kuhn-tet cavity"


def workload_config(args, p=None, prec_name="fp64"):
    """The configured workload at its full size (element and node counts of
    `p`, else from the mesh generator's formulas)."""
    n = args.n
    if args.config == "channel":
        E, N = (p.n_elems, p.n_nodes) if p is not None else (4 * n ** 3, (4 * n + 1) * (n + 1) ** 2)
    else:
        E, N = (p.n_elems, p.n_nodes) if p is not None else (6 * n ** 3, (n + 1) ** 3)
    if args.config == "channel":
        w = (f"SUPG hexa8 channel [0,4]x[0,1]^2, {4 * n}x{n}x{n} cells ({E} hexa, {N} nodes), "
             f"jitter 0.05h, parabolic inlet peak 1, mu=0.005, CFL 0.2, EXOPTS 1 0 1 1 1 1, {prec_name} form")
    else:
        if args.config == "cavity":
            kind, dtrule = "VMS", "invEps=400, nu=0.01, dt from CFL 0.2 on lid+sqrt(invEps)"
        else:
            kind, dtrule = "SUPG (EXOPTS 1 0 1 1 1 1)", "alpha=1, cI=4, nu=0.01, dt from CFL 0.05 on the lid speed"
        w = (f"{kind} tet4 lid-driven cavity {n}^3 cells x 6 Kuhn tets ({E} tets, {N} nodes), "
             f"{dtrule}, {prec_name} form")
    return {"workload": w, "elements": E, "nodes": N, "l2": "inputs larger than L2 (no flush)",
            "parallelism": "one independent problem per GPU"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=0, help="mesh size (default 96 for cavity/supg, 64 for channel)")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--config", default="cavity",
                    choices=["cavity", "supg", "channel", "batched", "serve", "partitioned", "poisson", "io"])
    ap.add_argument("--rates", default="10,30,100,1000", help="serve: arrival rates, requests/s")
    ap.add_argument("--requests", type=int, default=48, help="serve: requests per rate")
    ap.add_argument("--budget-gb", type=float, default=16.0, help="serve: HBM budget of the pooled batch")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ref-steps", type=int, default=5, help="reference arm: timed steps (bounded sample)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tile-elems", type=int, default=0)
    ap.add_argument("--tile-nodes", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0,
                    help="VMS register budget: tile kernel variant for this many resident CTAs an SM (0: default)")
    ap.add_argument("--graph-steps", type=int, default=0,
                    help="partitioned: iterations per captured CUDA graph (0: eager loop)")
    args = ap.parse_args()
    if not args.n:
        args.n = CONFIG_DEFAULT_N.get(args.config, 96)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    if args.config == "io":
        # host path: rank 0 reads (and, with a device, writes); no collective
        if rank == 0:
            print(json.dumps(io_line(args, world, run_io(args))), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    if args.config == "serve":
        if rank == 0:
            print(json.dumps(serve_line(args, run_serve(args, local_rank))), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.config == "partitioned":
        precs = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
        runs = {pn: run_partitioned(args, rank, world, local_rank, dist, pn) for pn in precs}
        if rank == 0:
            print(json.dumps(partitioned_line(args, world, runs)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.config == "poisson":
        rp = run_poisson(args, rank, world, local_rank, dist)
        if rank == 0:
            print(json.dumps(poisson_line(args, world, rp)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.config == "batched":
        rb = run_batched(args, rank, world, local_rank, dist)
        if rank == 0:
            print(json.dumps(batched_line(args, world, rb)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    # FP64 (the reference's precision) is the headline; the mixed form beside it
    precs = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    runs = {}
    for pn in precs:
        a2 = argparse.Namespace(**vars(args))
        a2.precision = pn
        runs[pn] = run_ours(a2, rank, world, local_rank, dist)
    if rank == 0:
        peak, peak_kind = hbm_peak()

        def summary(pn, r):
            E, N = r["E"], r["N"]
            ab = algorithmic_bytes(E, N, pn, args.config)
            klaunch = max(1, r["klaunch"])
            tile_ms = r["kprof"]["tile"] / klaunch
            achieved = ab / (tile_ms * 1e-3) / 1e9
            kernel = "vms_tile_kernel" if args.config == "cavity" else "supg_tile_kernel"
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": measured_traffic(kernel, pn, E), "peak_source": peak_kind, "kernel": kernel,
                    "algorithmic_bytes_per_launch": ab, "avg_launch_ms": tile_ms,
                    "iface_kernel_avg_ms": r["kprof"]["iface"] / klaunch}
            if stored_geometry_bytes(E, pn, args.config):
                roof["stored_geometry_bytes_per_launch"] = stored_geometry_bytes(E, pn, args.config)
            if args.config in SUPG_FLOPS and pn == "fp64":
                # the SUPG element work is FP64-pipe bound: FLOP rate beside the bytes
                roof["fp64_tflops"] = SUPG_FLOPS[args.config] * E / (tile_ms * 1e-3) / 1e12
                roof["fp64_flops_per_element_step"] = SUPG_FLOPS[args.config]
            out = {"value": world * E * args.steps / (r["ms"] / 1e3), "ms_per_step": r["ms"] / args.steps,
                   "roofline": roof, "gpu_launches": r["launches"], "clocks": r["clocks"]}
            if "e2e_s" in r:
                k = r["e2e_steps"]
                out["e2e"] = {"value": E * k / r["e2e_s"], "unit": "element-steps/s",
                              "h2d_bytes_per_step": r["h2d"] / k, "d2h_bytes_per_step": r["d2h"] / k,
                              "steps": k,
                              "note": f"one whole {k}-step solve of the workload through the C ABI: problem "
                                      f"create + batch create (host layout, H2D of mesh and initial state) + "
                                      f"{k} steps + state readback (D2H), wall clock"}
            return out

        head = precs[0]
        r = runs[head]
        E, N = r["E"], r["N"]
        s = summary(head, r)
        line = {
            "metric": METRIC[args.config], "value": s["value"], "unit": "element-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": s["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": dict(workload_config(args, r["p"], head),
                           parallelism=f"{world} independent solve(s), one per GPU"),
            "roofline": s["roofline"],
            "gpu_launches": r["launches"], "clocks": r["clocks"], "layout": r["layout"],
        }
        if "e2e" in s:
            line["e2e"] = s["e2e"]
        if "mixed" in runs and head != "mixed":
            sm = summary("mixed", runs["mixed"])
            line["mixed"] = dict(sm, dtype="f32+f64")
            line["mixed_over_fp64"] = sm["value"] / s["value"]
            line["mixed_vs_fp64_rel_l2"] = accuracy_run(args, local_rank, 200)
        if world == 1 and not args.no_cpu:
            try:
                line["cpu_baseline"] = cpu_baseline(args)
            except Exception as e:  # the baseline is reported, not required
                line["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
