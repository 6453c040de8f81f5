"""Failure detection on the GPU without a GPU fault.

The reference's only failure exit is the SUPG EXITCOND check
(femSUPGExplicitFluidSolver.cpp:1635-1643); it has no device and no waits.
Here every wait of the VMS tile kernel (a CTA waiting for the bulk copies of
its next chunk of elements) is bounded.  The bound is a launch parameter, so
a test can make it run out: with a limit of 0 polls every wait gives up at
once, each CTA waits (bounded) for the copies it issued, leaves its nodes
untouched and sets FM_ERR_TIMEOUT, which the host reads from fm_batch_sync.
The context stays usable and the problem stays stopped at its last good
state."""
import numpy as np
import pytest

from femorph_b200 import api, mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [api.FM_FP64, api.FM_MIXED])
def test_chunk_wait_timeout_reported_state_untouched(precision):
    p = mesh.cavity(6, seed=3, steps=10)
    g = api.GpuProblem(p, precision)
    b = api.Batch([g], tile_elems=128)
    b.step(2)
    b.sync()
    u0, p0, _, sd0 = g.state()
    b.set_wait_limit(0)
    b.step(1)
    with pytest.raises(api.FmError) as ei:
        b.sync()
    assert ei.value.code == api.FM_ERR_TIMEOUT
    assert g.status() == api.FM_ERR_TIMEOUT
    u1, p1, _, sd1 = g.state()
    assert np.array_equal(u0, u1) and np.array_equal(p0, p1) and np.array_equal(sd0, sd1)
    # a problem with a device error stays stopped, even with the wait restored
    b.set_wait_limit(1 << 22)
    b.step(2)
    with pytest.raises(api.FmError):
        b.sync()
    u2, p2, _, _ = g.state()
    assert np.array_equal(u0, u2) and np.array_equal(p0, p2)
    b.close()
    g.close()


def test_device_usable_after_timeout():
    """After a timed-out launch the device context is intact: new batches of
    the same problem run and give identical results."""
    p = mesh.cavity(5, seed=8, steps=6)
    g = api.GpuProblem(p)
    b = api.Batch([g])
    b.set_wait_limit(0)
    b.step(1)
    with pytest.raises(api.FmError) as ei:
        b.sync()
    assert ei.value.code == api.FM_ERR_TIMEOUT
    b.close()
    g.close()
    ref = []
    for _ in range(2):
        g = api.GpuProblem(p)
        b = api.Batch([g])
        b.step(6)
        b.sync()
        ref.append(g.state(elements=False)[:2])
        b.close()
        g.close()
    assert np.array_equal(ref[0][0], ref[1][0]) and np.array_equal(ref[0][1], ref[1][1])
