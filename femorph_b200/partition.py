"""One mesh split over several GPUs: one process per GPU, one exchange per
dual iteration (VMS) or step (SUPG).

Every process builds the whole problem on the host (BCs resolved and lumped
masses formed on the whole mesh), keeps the part with its rank's index and
advances it on its GPU.  Between the two halves of each iteration the
parts' partial sums at the shared nodes are added with one
``torch.distributed.all_reduce`` (NCCL over NVLink / NVSwitch) on a packed
buffer of 4 doubles per shared node; every part then updates its own copy of
each shared node from the same sum, so the copies stay bit-identical.

The reference solves a mesh in one process (femVMSExplicitFluidSolver::solve,
src/femVMSExplicitFluidSolver.cpp:842-1334; femSUPGExplicitFluidSolver::solve,
src/femSUPGExplicitFluidSolver.cpp:794-1735); a partitioned run computes the
same per-element terms and the same nodal updates, with the nodal sums of
shared nodes formed in a different order (FP64 rounding differences only).
"""
from __future__ import annotations

import numpy as np

from . import api
from . import mesh as _mesh


def assemble(n_nodes: int, n_elems: int, parts):
    """Whole-mesh (u (N,3), p) from per-part results [(GpuPart-like, u, p)]:
    node values from any part holding the node (shared copies are equal),
    element values (SUPG pressure) from the owning part."""
    u = np.zeros((n_nodes, 3))
    vms = None
    for part, pu, pp in parts:
        u[part.node_global] = pu
        vms = part.solver == _mesh.VMS
    p = np.zeros(n_nodes if vms else n_elems)
    for part, pu, pp in parts:
        if vms:
            p[part.node_global] = pp
        else:
            p[part.elem_global] = pp
    return u, p


class PartitionedSolve:
    """This rank's part of ``problem`` split over the default process group.

    ``step(n)`` advances the whole mesh by n time steps; every rank calls it
    with the same n.  ``elem_part`` overrides the default split (Morton bands
    of equal element count).  ``graph_steps`` > 0 records that many
    iterations (tile kernel, partial sums, all-reduce, shared-node update) in
    one CUDA graph and replays it, so the host issues one launch per
    ``graph_steps`` iterations instead of four calls per iteration."""

    def __init__(self, problem: "_mesh.Problem", precision: int = api.FM_FP64, device: int | None = None,
                 elem_part=None, tile_elems: int = 0, tile_nodes: int = 0, threads: int = 0,
                 graph_steps: int = 0):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank = dist.get_rank() if dist.is_initialized() else 0
        self.world = dist.get_world_size() if dist.is_initialized() else 1
        self.device = torch.cuda.current_device() if device is None else device
        self.n_nodes, self.n_elems = problem.n_nodes, problem.n_elems
        full = api.GpuProblem(problem, precision)
        self.part = full.part(self.world, self.rank, elem_part)
        full.close()
        self.batch = api.Batch([self.part], tile_elems=tile_elems, tile_nodes=tile_nodes, threads=threads,
                               device=self.device)
        send, recv, self.count = self.batch.exchange_buffers()
        dev = torch.device("cuda", self.device)
        self.send = torch.as_tensor(send, device=dev)
        self.recv = torch.as_tensor(recv, device=dev)
        self.per_step = self.batch.iterations_per_step()
        # the library's kernels, the copy and the all-reduce share one stream
        # (a NULL stream would mean the batch's own stream to the library)
        self.stream = torch.cuda.Stream(device=self.device)
        self.graph_steps = int(graph_steps)
        self.graph = None
        self.iterations = 0

    def _iteration(self) -> None:
        s = self.stream.cuda_stream
        self.batch.exchange_begin(s)
        if self.world > 1:
            self.recv.copy_(self.send)
            self.dist.all_reduce(self.recv)
        self.batch.exchange_end(s)

    def iterate(self) -> None:
        """One dual iteration (VMS) / step (SUPG) of this part: tile kernel and
        partial sums, the all-reduce, the shared-node update."""
        with self.torch.cuda.stream(self.stream):
            self._iteration()
        self.iterations += 1

    def _capture(self) -> None:
        # recorded on this part's stream after at least one eager iteration
        # (which opened the library's device targets and set up NCCL)
        g = self.torch.cuda.CUDAGraph()
        with self.torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
            for _ in range(self.graph_steps):
                self._iteration()
        self.graph = g

    def prepare_graph(self) -> None:
        """Records the graph now (runs one eager iteration first if none has
        run), so that later steps only replay it."""
        if self.graph_steps > 0 and self.graph is None:
            if self.iterations == 0:
                self.iterate()
            self._capture()

    def step(self, n: int = 1) -> None:
        left = int(n) * self.per_step
        if self.graph_steps > 0:
            if self.graph is None and left > self.graph_steps:
                if self.iterations == 0:
                    self.iterate()
                    left -= 1
                self._capture()
            while self.graph is not None and left >= self.graph_steps:
                with self.torch.cuda.stream(self.stream):
                    self.graph.replay()
                self.batch.exchange_account(self.graph_steps)
                self.iterations += self.graph_steps
                left -= self.graph_steps
        for _ in range(left):
            self.iterate()

    def sync(self) -> None:
        self.stream.synchronize()
        self.batch.sync()

    def local_state(self):
        u, p, _, _ = self.part.state(elements=False)
        return u, p

    def gather_state(self):
        """Whole-mesh (u, p) on rank 0 (None on the other ranks)."""
        u, p = self.local_state()
        mine = (self.part.node_global, self.part.elem_global, self.part.solver, u, p)
        if self.world == 1:
            got = [mine]
        else:
            got = [None] * self.world if self.rank == 0 else None
            self.dist.gather_object(mine, got, dst=0)
        if self.rank != 0:
            return None

        class _P:
            pass
        parts = []
        for ng, eg, solver, pu, pp in got:
            q = _P()
            q.node_global, q.elem_global, q.solver = ng, eg, solver
            parts.append((q, pu, pp))
        return assemble(self.n_nodes, self.n_elems, parts)

    def close(self) -> None:
        """Releases the graph (before any process-group teardown), the batch
        and the part."""
        self.graph = None
        self.batch.close()
        self.part.close()
