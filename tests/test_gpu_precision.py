"""16-bit moment storage against a committed FP64 solution.

The periodic Taylor-Green vortex, D3Q27, 128^3, Re 400, u0 0.04, 1000 steps:
at this Reynolds number tau - 1/2 = 0.0061, the value of the 512^3 vortex at
Re 1600, so the rounding noise 16-bit storage adds to the stored moments each
step is damped as weakly as in that configuration.  The FP64 reference
(tests/golden/tgv128re400_fp64.npz, made by tests/golden/make_tgv_fixtures.py
with the FP64 oracle) holds 3u on z planes 0, 40 and 80.

Bound: the relative L2 error of the velocity against FP64 must be at most
1e-3 for the split-velocity fp16 storage (MRLBM_F16U).  Plain fp16 storage
(3u rounded to 11 significant bits each step) is measured and reported, and
FP32 storage must stay within 1e-4.
"""
import os

import numpy as np
import pytest

import mrlbm

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def run(storage):
    ref = np.load(os.path.join(HERE, "golden", "tgv128re400_fp64.npz"))
    n, steps, re = int(ref["n"]), int(ref["steps"]), float(ref["re"])
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * 0.04 * L / re
    assert abs(tau - float(ref["tau"])) < 1e-12
    d = mrlbm.make_desc(n, n, n, lattice=27, storage=storage, tau=tau)
    dom = mrlbm.Domain(d)
    dom.init_taylor_green(0.04, L)
    dom.step(steps)
    m = dom.moments()
    dom.close()
    planes = [int(p) for p in ref["planes"]]
    g = np.moveaxis(m[1:4][:, planes].astype(np.float64), 0, -1)
    o = ref["u3"].astype(np.float64)
    return float(np.sqrt(np.sum((g - o) ** 2) / np.sum(o ** 2)))


def test_split_velocity_fp16_storage_within_1e3_of_fp64():
    e16u = run(mrlbm.F16U)
    e16 = run(mrlbm.F16)
    e32 = run(mrlbm.F32)
    print("TGV 128^3 Re 400, 1000 steps, u rel L2 vs FP64: fp32 %.2e, fp16 %.2e, fp16 split velocity %.2e"
          % (e32, e16, e16u))
    assert e32 < 1e-4
    assert e16u <= 1e-3


def test_split_velocity_round_trip_keeps_velocity_to_fp32_level():
    n = 24
    d = mrlbm.make_desc(n, n, n, lattice=19, storage=mrlbm.F16U, tau=0.6)
    dom = mrlbm.Domain(d)
    rng = np.random.default_rng(3)
    rho = 1 + 0.001 * rng.standard_normal((n, n, n))
    u = 0.04 * rng.standard_normal((3, n, n, n))
    dom.init_flow(rho, u[0], u[1], u[2])
    m = dom.moments()
    # 3u keeps ~22 significant bits (plain fp16: 11)
    np.testing.assert_allclose(m[1:4] / 3.0, u, rtol=2e-6, atol=1e-9)
    dom.set_moments(m)
    np.testing.assert_allclose(dom.moments()[1:4], m[1:4], rtol=1e-6, atol=1e-10)
    dom.close()
