"""The element kernels' own reciprocal, inverse cube root and square root
(fm_device.cuh: a correction step from the PTX approximate FP32 seeds,
Newton's / Householder's published methods) against CUDA's 1.0/x, rcbrt,
sqrt and rcbrtf on the same device, over a sweep that crosses the 1e-37 / 1e37 switch points to CUDA's
own operations, with ulp bounds.  (The reference computes these on the host:
1.0 / detJ, pow(6V, 1/3), sqrt - src/femVMSExplicitFluidSolver.cpp:64, 75,
585.)"""
import numpy as np
import pytest

from femorph_b200 import api

pytestmark = pytest.mark.gpu


def ulps(a, b, dtype=np.float64):
    a = np.asarray(a, dtype)
    b = np.asarray(b, dtype)
    return np.abs(a - b) / np.spacing(np.abs(b).astype(dtype))


def sweep():
    rng = np.random.default_rng(5)
    x = [10.0 ** rng.uniform(-40, 40, 200000), rng.uniform(0.5, 2.0, 50000),
         10.0 ** rng.uniform(-12, 2, 50000)]
    for edge in (1e-37, 1e37):
        x.append(edge * (1 + np.linspace(-1e-6, 1e-6, 41)))
        x.append(np.array([np.nextafter(edge, 0), edge, np.nextafter(edge, np.inf)]))
    x.append(np.array([1.0, 2.0, 3.0, 8.0, 27.0, 1.0 / 6.0, 1e-300, 1e300]))
    return np.concatenate(x)


def test_newton_raphson_math_within_ulps_of_cuda():
    x = sweep()
    x = np.concatenate([x, -x[:1000]])            # the reciprocal takes negative values too
    out = np.zeros((x.size, 8))
    api.check(api.lib().fm_math_check(x.ctypes.data, x.size, out.ctypes.data))
    pos = x > 0
    r_rcp = ulps(out[:, 0], out[:, 1]).max()
    r_cbrt = ulps(out[pos, 2], out[pos, 3]).max()
    r_sqrt = ulps(out[pos, 4], out[pos, 5]).max()
    # FP32 form over the FP32 normal range
    f = pos & (x > 1e-30) & (x < 1e30)
    r_cbrtf = ulps(out[f, 6], out[f, 7], np.float32).max()
    # against extended-precision values on the host (CUDA's rcbrt is itself
    # within about an ulp)
    ld = np.asarray(x[pos], np.longdouble)
    exact = np.asarray(ld ** (np.longdouble(-1) / np.longdouble(3)), np.float64)
    r_cbrt_exact = ulps(out[pos, 2], exact).max()
    print(f"[math] max ulps: rcp_nr vs 1/x {r_rcp:.2f}, rcbrt_nr vs rcbrt {r_cbrt:.2f} "
          f"(vs extended {r_cbrt_exact:.2f}), sqrt_nr vs sqrt {r_sqrt:.2f}, rcbrt_nr(float) vs rcbrtf {r_cbrtf:.2f}")
    assert r_rcp <= 1.0, r_rcp
    assert r_sqrt <= 1.0, r_sqrt
    assert r_cbrt <= 2.0 and r_cbrt_exact <= 2.0, (r_cbrt, r_cbrt_exact)
    assert r_cbrtf <= 4.0, r_cbrtf
    # exact cases
    i1 = np.nonzero(x == 1.0)[0][0]
    i8 = np.nonzero(x == 8.0)[0][0]
    assert out[i1, 0] == 1.0 and out[i1, 4] == 1.0
    assert abs(out[i8, 2] - 0.5) <= np.spacing(0.5)
