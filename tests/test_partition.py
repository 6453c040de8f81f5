"""Partitioned single mesh: host logic on CPU (no GPU needed).

A mesh split into parts: the parts own every element exactly once, carry the
whole mesh's masses and BC records at their nodes, and agree on one
exchange list.  The exchange itself is checked with world size 2 over gloo:
each rank assembles a nodal sum over its own elements, packs its shared
nodes by exchange index, all-reduces, and must then hold the whole mesh's
sum at every node it has, which is what the GPU exchange relies on.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from femorph_b200 import api, mesh


def _parts(p, n, elem_part=None):
    full = api.GpuProblem(p)
    parts = [full.part(n, k, elem_part) for k in range(n)]
    return full, parts


def _shared(p, ep):
    """Nodes touched by more than one part (numpy restatement)."""
    npe = p.elem_type
    conn = np.asarray(p.conn).reshape(-1, npe)
    lo = np.full(p.n_nodes, 1 << 30)
    hi = np.full(p.n_nodes, -1)
    for a in range(npe):
        np.minimum.at(lo, conn[:, a], ep)
        np.maximum.at(hi, conn[:, a], ep)
    return (hi >= 0) & (lo != hi)


@pytest.mark.parametrize("case", ["vms", "supg_hexa"])
@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_parts_cover_the_mesh(case, n):
    p = mesh.cavity(6, seed=1) if case == "vms" else mesh.channel(8, 4, 3, seed=2, steps=4)
    full, parts = _parts(p, n)
    ep = full.partition_elements(n)
    assert ep.min() == 0 and ep.max() == n - 1
    counts = np.bincount(ep, minlength=n)
    assert counts.max() - counts.min() <= 1                       # equal bands
    owned = np.concatenate([q.elem_global for q in parts])
    assert np.array_equal(np.sort(owned), np.arange(p.n_elems))   # each element once
    shared = _shared(p, ep)
    xset = shared.copy()
    if p.solver == mesh.VMS:
        xset[:4] = True
    xlist = np.flatnonzero(xset)
    fm = full.mass()
    npe = p.elem_type
    conn = np.asarray(p.conn).reshape(-1, npe)
    for k, q in enumerate(parts):
        assert q.part_index == k and q.n_parts == n and q.x_total == len(xlist)
        assert np.all(np.diff(q.node_global) > 0)                 # global order
        touched = np.unique(conn[ep == k])
        want = np.union1d(touched, np.arange(4)) if p.solver == mesh.VMS else touched
        assert np.array_equal(q.node_global, want)
        # exchange index = position in the global shared list
        assert np.array_equal(q.xidx >= 0, xset[q.node_global])
        assert np.array_equal(xlist[q.xidx[q.xidx >= 0]], q.node_global[q.xidx >= 0])
        # whole-mesh masses at the part's nodes
        m = q.mass()
        if p.solver == mesh.VMS:
            assert np.array_equal(m, fm[q.node_global])
        else:
            assert np.array_equal(m.reshape(-1, 3), fm.reshape(-1, 3)[q.node_global])
    for q in parts:
        q.close()
    full.close()


def test_custom_split_and_errors():
    p = mesh.cavity(4, seed=3)
    full = api.GpuProblem(p)
    ep = (np.arange(p.n_elems) % 2).astype(np.int32)              # checkerboard-like split
    q = full.part(2, 1, ep)
    assert np.array_equal(q.elem_global, np.flatnonzero(ep == 1))
    with pytest.raises(api.FmError):
        full.part(2, 2)                                           # part out of range
    with pytest.raises(api.FmError):
        full.part(2, 0, np.full(p.n_elems, 3, np.int32))          # bad part ids
    with pytest.raises(api.FmError):
        full.part(2, 1, np.zeros(p.n_elems, np.int32))            # empty part
    with pytest.raises(api.FmError):
        q.part(2, 0)                                              # parts are not split again
    q.close()
    full.close()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _nodal_sum(coords, conn):
    """Per node: sum over incident elements of (V/4, centroid x, y, z)."""
    x = coords[conn]                                   # (E, npe, 3)
    cen = x.mean(axis=1)
    d = x[:, 1:4] - x[:, :1]
    vol = np.abs(np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2]))) / 6.0
    vals = np.concatenate([vol[:, None] / 4.0, cen], axis=1)   # (E, 4)
    out = np.zeros((coords.shape[0], 4))
    for a in range(conn.shape[1]):
        np.add.at(out, conn[:, a], vals)
    return out


def _exchange_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p = mesh.cavity(7, seed=5)
    full = api.GpuProblem(p)
    part = full.part(world, rank)
    coords = np.asarray(p.coords).reshape(-1, 3)[part.node_global]
    conn = np.asarray(p.conn).reshape(-1, 4)[part.elem_global]
    # local numbering of the part's connectivity
    loc = np.full(p.n_nodes, -1)
    loc[part.node_global] = np.arange(part.n_nodes)
    local = _nodal_sum(coords, loc[conn])
    buf = torch.zeros(part.x_total * 4, dtype=torch.float64)
    sh = part.xidx >= 0
    buf.view(-1, 4)[torch.as_tensor(part.xidx[sh], dtype=torch.long)] = torch.as_tensor(local[sh])
    dist.all_reduce(buf)
    done = local.copy()
    done[sh] = buf.view(-1, 4).numpy()[part.xidx[sh]]
    whole = _nodal_sum(np.asarray(p.coords).reshape(-1, 3), np.asarray(p.conn).reshape(-1, 4))
    err = float(np.abs(done - whole[part.node_global]).max() / np.abs(whole).max())
    q.put((rank, err, int(sh.sum()), part.x_total))
    dist.barrier()
    dist.destroy_process_group()


def test_exchange_two_ranks_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = sorted(q.get(timeout=180) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, err, nsh, xt in out:
        assert err < 1e-14, (rank, err)
        assert 4 < nsh <= xt
    assert out[0][3] == out[1][3]
