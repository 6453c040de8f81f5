"""Partitioned single mesh on the GPU: a mesh split into parts, each part an
ordinary tiled problem, one exchange of the shared nodes' partial sums per
dual iteration (VMS) or step (SUPG).

Results must equal the unsplit mesh's up to the rounding of the reordered
nodal sums: relative L2 <= 1e-11 after 20 steps in FP64 (the same bar as
the FP64 parity tests, 1e-12 per step).  Runs on one GPU: all parts in one
batch (the exchange is a plain sum over the parts' slices), two batches
whose exchange is summed by torch between the halves of each iteration (the
multi-process protocol, driven from one thread), and the torch.distributed
driver with an NCCL group of one process.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from femorph_b200 import api, mesh
from femorph_b200.partition import assemble
from oracle import oracle_b

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def whole(p, steps, precision=api.FM_FP64):
    g = api.GpuProblem(p, precision)
    b = api.Batch([g])
    b.step(steps)
    b.sync()
    u, pr, _, _ = g.state(elements=False)
    b.close()
    g.close()
    return u, pr


def split_one_batch(p, n, steps, precision=api.FM_FP64, elem_part=None):
    full = api.GpuProblem(p, precision)
    parts = [full.part(n, k, elem_part) for k in range(n)]
    b = api.Batch(parts)
    b.step(steps)
    b.sync()
    res = [(q, *q.state(elements=False)[:2]) for q in parts]
    # copies of a shared node are bit-identical on every part
    seen = {}
    for q, u, _ in res:
        for gid, row in zip(q.node_global[q.xidx >= 0], u[q.xidx >= 0]):
            if gid in seen:
                assert np.array_equal(seen[gid], row)
            seen[gid] = row
    out = assemble(p.n_nodes, p.n_elems, res)
    b.close()
    for q in parts:
        q.close()
    full.close()
    return out


@pytest.mark.parametrize("n", [2, 3, 4])
def test_vms_parts_in_one_batch_match_whole_mesh(n):
    p = mesh.cavity(12, seed=7, steps=20)
    u0, p0 = whole(p, 20)
    u1, p1 = split_one_batch(p, n, 20)
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL, (rel(u1, u0), rel(p1, p0))


def test_vms_dual_iterations_and_mixed():
    p = mesh.cavity(10, seed=8, steps=10)
    p.tot_dual_steps = 2
    u0, p0 = whole(p, 10)
    u1, p1 = split_one_batch(p, 3, 10)
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL
    q = mesh.cavity(10, seed=9, steps=20)
    u0, p0 = whole(q, 20, api.FM_MIXED)
    u1, p1 = split_one_batch(q, 2, 20, api.FM_MIXED)
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL


def test_supg_hexa_ab2_bbar_parts():
    p = mesh.channel(12, 5, 4, seed=3, steps=20, ex_opts=(0, 1, 1, 1, 1, 1))
    u0, p0 = whole(p, 20)
    u1, p1 = split_one_batch(p, 3, 20)
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL, (rel(u1, u0), rel(p1, p0))


def test_supg_tet_custom_split():
    p = mesh.cavity(8, seed=4, steps=20, solver=mesh.SUPG, cfl=0.05)
    ep = (np.arange(p.n_elems) * 7 % 3).astype(np.int32)     # scattered parts: many shared nodes
    u0, p0 = whole(p, 20)
    u1, p1 = split_one_batch(p, 3, 20, elem_part=ep)
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL


def test_vms_parts_against_oracle():
    """The split solve (3 Morton-band parts, one exchange per iteration)
    against the oracle directly: FP64 within 1e-10 after 40 steps."""
    p = mesh.cavity(16, seed=5, steps=40)
    o = oracle_b.OracleSolve(p)
    o.step(40)
    st = o.state()[0]
    u1, p1 = split_one_batch(p, 3, 40)
    eu, ep = rel(u1, st[:, :3]), rel(p1, st[:, 3])
    print(f"[parity] vms16 in 3 parts, step 40 vs oracle: u {eu:.3e} p {ep:.3e}")
    assert eu <= 1e-10 and ep <= 1e-10, (eu, ep)


def test_supg_hexa_parts_against_oracle():
    """SUPG hexa8 (AB2, B-bar) split in 3 parts against the oracle: velocity
    and element pressure within 1e-10 after 20 steps."""
    p = mesh.channel(16, 6, 5, seed=6, steps=20, ex_opts=(0, 1, 1, 1, 1, 1))
    o = oracle_b.OracleSolve(p)
    o.step(20)
    st, oel, _, _ = o.state()
    u1, p1 = split_one_batch(p, 3, 20)
    eu, ep = rel(u1, st[:, :3]), rel(p1, oel[:, 0])
    print(f"[parity] channel16x6x5 in 3 parts, step 20 vs oracle: u {eu:.3e} element p {ep:.3e}")
    assert eu <= 1e-10 and ep <= 1e-10, (eu, ep)


def test_two_batches_external_exchange():
    """The multi-process protocol on one GPU: each batch holds one of two
    parts; between exchange_begin and exchange_end the two send buffers are
    summed into both recv buffers (what an all-reduce does)."""
    import torch
    p = mesh.cavity(12, seed=11, steps=15)
    u0, p0 = whole(p, 15)
    full = api.GpuProblem(p)
    parts = [full.part(2, k) for k in range(2)]
    bs = [api.Batch([q]) for q in parts]
    with pytest.raises(api.FmError):
        bs[0].step(1)                     # the other part lives elsewhere
    bufs = []
    for b in bs:
        s, r, n = b.exchange_buffers()
        bufs.append((torch.as_tensor(s, device="cuda"), torch.as_tensor(r, device="cuda")))
    # one ordinary stream for the library's kernels and torch's sum (the
    # library reads a NULL stream as "the batch's own stream", so torch's
    # legacy default stream, handle 0, cannot be passed)
    ts = torch.cuda.Stream()
    stream = ts.cuda_stream
    with torch.cuda.stream(ts):
        for _ in range(15 * bs[0].iterations_per_step()):
            for b in bs:
                b.exchange_begin(stream)
            tot = bufs[0][0] + bufs[1][0]
            for _, r in bufs:
                r.copy_(tot)
            for b in bs:
                b.exchange_end(stream)
    torch.cuda.synchronize()
    for b in bs:
        b.sync()
    u1, p1 = assemble(p.n_nodes, p.n_elems, [(q, *q.state(elements=False)[:2]) for q in parts])
    assert rel(u1, u0) < TOL and rel(p1, p0) < TOL, (rel(u1, u0), rel(p1, p0))
    with pytest.raises(api.FmError):
        bs[0].exchange_end(stream)        # end without begin
    for b in bs:
        b.close()
    for q in parts:
        q.close()
    full.close()


def test_batch_rules_for_parts():
    p = mesh.cavity(6, seed=12, steps=3)
    full = api.GpuProblem(p)
    other = api.GpuProblem(mesh.cavity(5, seed=13))
    a, b = full.part(2, 0), full.part(2, 1)
    with pytest.raises(api.FmError):
        api.Batch([a, other])             # parts take no other problems
    with pytest.raises(api.FmError):
        api.Batch([a, full.part(2, 0)])   # the same part twice
    bt = api.Batch([a, b])
    with pytest.raises(api.FmError):
        bt.step_ragged([1, 2])            # parts advance together
    bt.step(2)
    bt.sync()
    bt.close()


def test_partitioned_solve_graph_replay_equals_eager():
    """One process, one part: the CUDA-graph replay of the exchange loop gives
    the same state, bit for bit, as the eager loop, and the library counts
    the replayed steps."""
    from femorph_b200.partition import PartitionedSolve
    p = mesh.cavity(10, seed=23, steps=17)
    out = []
    for gs in (0, 4):
        s = PartitionedSolve(p, graph_steps=gs)
        s.step(9)
        s.step(8)
        s.sync()
        out.append(s.gather_state())
        nn = C_steps(s.part)
        assert nn == 17, nn
        s.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def C_steps(part):
    import ctypes as C
    st = C.c_int64()
    api.check(api.lib().fm_problem_info(part.h, None, None, None, None, C.byref(st)))
    return st.value


DRIVER = r"""
import os, sys, json
import numpy as np, torch, torch.distributed as dist
sys.path.insert(0, os.getcwd())
from femorph_b200 import api, mesh
from femorph_b200.partition import PartitionedSolve
os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
dist.init_process_group("nccl", rank=0, world_size=1)
torch.cuda.set_device(0)
p = mesh.cavity(10, seed=21, steps=12)
s = PartitionedSolve(p, graph_steps=int(os.environ.get("GRAPH_STEPS", "0")))
s.step(12)
s.sync()
u, pr = s.gather_state()
g = api.GpuProblem(p); b = api.Batch([g]); b.step(12); b.sync()
u0, p0, _, _ = g.state(elements=False)
print(json.dumps(dict(du=float(np.linalg.norm(u - u0) / np.linalg.norm(u0)),
                      dp=float(np.linalg.norm(pr - p0) / np.linalg.norm(p0)), x=int(s.count))))
s.close(); b.close(); g.close()
dist.destroy_process_group()
"""


@pytest.mark.parametrize("graph_steps", [0, 5])
def test_torch_distributed_driver_nccl_one_rank(tmp_path, graph_steps):
    import json
    import socket
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0",
               GRAPH_STEPS=str(graph_steps))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", DRIVER], cwd=root, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["du"] < TOL and out["dp"] < TOL, out
    assert out["x"] == 16                 # one part: the exchange list is nodes 0..3
