"""Host-side checks of the tile layout the kernels rely on
(fm_problem_check_layout): local connectivity, interior nodes touched by one
tile only, colours without shared nodes, incidence lists in element order,
interface slots in tile order, every element and node once, shared nodes of
partition parts on interface entries - over the mesh families, tile sizes
and precisions the solvers use (the mixed form flags
FP64-Jacobian elements in the local connectivity; the interface nodes are
reordered to balance the owner threads).  No GPU needed."""
import pytest

from femorph_b200 import api, mesh

CASES = [
    ("vms-cavity", lambda: mesh.cavity(10, seed=1, steps=2), api.FM_FP64, {}),
    ("vms-cavity-mixed", lambda: mesh.cavity(10, seed=1, steps=2), api.FM_MIXED, {}),
    ("vms-cavity-small-tiles", lambda: mesh.cavity(12, seed=2, steps=2), api.FM_FP64,
     dict(tile_elems=384, tile_nodes=160)),
    ("vms-cavity-large-tiles", lambda: mesh.cavity(16, seed=2, steps=2), api.FM_FP64,
     dict(tile_elems=2048, tile_nodes=512)),
    ("supg-tet", lambda: mesh.cavity(8, seed=4, steps=2, solver=mesh.SUPG, cfl=0.05), api.FM_FP64, {}),
    ("supg-hexa", lambda: mesh.channel(24, 8, 8, seed=3, steps=2), api.FM_FP64, {}),
    ("supg-hexa-mixed", lambda: mesh.channel(24, 8, 8, seed=3, steps=2), api.FM_MIXED, {}),
    ("batched-member", lambda: mesh.batched_cavities(4, seed=7, n_lo=5, n_hi=9)[2], api.FM_FP64, {}),
]


@pytest.mark.parametrize("name,make,prec,tune", CASES, ids=[c[0] for c in CASES])
def test_layout_invariants(name, make, prec, tune):
    g = api.GpuProblem(make(), prec)
    g.check_layout(**tune)
    g.close()


@pytest.mark.parametrize("solver,n_parts", [(mesh.VMS, 2), (mesh.VMS, 3), (mesh.SUPG, 4)])
def test_layout_invariants_partition_parts(solver, n_parts):
    """Every part of a split mesh: the same invariants, and its shared nodes
    are interface nodes carrying their exchange index."""
    g = api.GpuProblem(mesh.cavity(10, seed=5, steps=2, solver=solver, cfl=0.05))
    for k in range(n_parts):
        part = g.part(n_parts, k)
        assert (part.xidx >= 0).any()
        part.check_layout()
        part.check_layout(tile_elems=256, tile_nodes=128)
        part.close()
    g.close()
