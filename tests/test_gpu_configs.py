"""The benchmark configurations at their own sizes against the FP64 oracle.

* Lid-driven cavity 64^3, D3Q19, Re 100, lid 0.05, 2000 steps (the
  lidDrivenCavity_3D case, src/cases/lidDrivenCavity_3D/constants.inc:35-36):
  every stored moment against the FP64 oracle run on the host at full size,
  within the per-moment bounds of the lid-cavity test of test_gpu_parity.py
  (rho and u: relative L2 5e-5, Linf 5e-4; second moments 3e-4 / 2e-3) or
  twice the error of the oracle's own FP32 build, whichever is larger (a
  driven flow accumulates FP32 round-off over its 2000 steps).
* Periodic Taylor-Green vortex 256^3, D3Q27, Re 1600, u0 0.04, 1000 steps
  (src/cases/taylorGreen/constants.inc:14-16): the kinetic energy every 100
  steps and every stored moment on z planes 0 and 96 (every 4th node in x and
  y) against the FP64 oracle's values in tests/golden/tgv256_fp64.npz (made by
  tests/golden/make_tgv_fixtures.py), with the per-moment bounds of
  test_gpu_parity.py.
* FP16 batch members: three uneven FP16 lid cavities advanced together by the
  batched kernel, each against the FP64 oracle.
* An FP16 power-law duct request (voxel obstacles, body force) solved by the
  server, against the FP64 oracle on the description and node types the
  server built for it (mrlbm_request_describe).

16-bit storage rounds every stored moment each step, so its bounds are the
measured 16-bit error level with a margin, stated next to each assertion.
"""
import os

import numpy as np
import pytest

import mrlbm
import parity_util as pu

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def per_moment_bounds(res, yard, l2=2e-5, linf=2e-4, l2_2=3e-4, linf_2=2e-3):
    bad = []
    for k, (e2, einf) in res.items():
        a2, ainf = (l2_2, linf_2) if 4 <= k <= 9 else (l2, linf)
        a2, ainf = max(a2, 2 * yard[k][0]), max(ainf, 2 * yard[k][1])
        if not (e2 <= a2 and einf <= ainf):
            bad.append("moment %d: rel L2 %.3e (bound %.2e), rel Linf %.3e (bound %.2e)" % (k, e2, a2, einf, ainf))
    return bad


def test_lid_cavity_64_full_run_matches_fp64_oracle():
    n, steps = 64, 2000
    d = mrlbm.lid_cavity_desc(n, re=100.0, lid_u=0.05)
    nt = mrlbm.lid_cavity_node_types(n, n, n, 1)
    dom = mrlbm.Domain(d)
    dom.set_node_types(nt)
    dom.init_uniform()
    m0 = pu.gpu_to_oracle_layout(dom.moments())
    dom.step(steps)
    g = dom.moments()
    dom.close()
    o64 = pu.oracle_for(d, nt)
    o64.set_moments(m0)
    o64.step(steps)
    o = o64.moments()
    o32 = pu.oracle_for(d, nt, fp32=True)
    o32.set_moments(m0)
    o32.step(steps)
    yard = pu.compare(np.moveaxis(o32.moments(), -1, 0), o)
    res = pu.compare(g, o)
    for k in range(10):
        print("C1 moment %d: GPU rel L2 %.2e Linf %.2e | FP32 oracle %.2e %.2e" % (k, *res[k], *yard[k]))
    assert pu.velocity_rel_l2(g, o) < 1e-4
    bad = per_moment_bounds(res, yard, l2=5e-5, linf=5e-4)
    assert not bad, "; ".join(bad)


def test_taylor_green_256_d3q27_matches_fp64_fixture():
    ref = np.load(os.path.join(HERE, "golden", "tgv256_fp64.npz"))
    n, steps, re = int(ref["n"]), int(ref["steps"]), float(ref["re"])
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * 0.04 * L / re
    assert abs(tau - float(ref["tau"])) < 1e-12
    d = mrlbm.make_desc(n, n, n, lattice=27, tau=tau)
    dom = mrlbm.Domain(d)
    dom.init_taylor_green(0.04, L)
    ke = [dom.sums()["kinetic_energy"]]
    for _ in range(steps // 100):
        dom.step(100)
        ke.append(dom.sums()["kinetic_energy"])
    m = dom.moments()
    dom.close()
    ke_ref = ref["ke"][:, 1]
    ke_err = np.abs(np.array(ke) - ke_ref) / ke_ref
    print("TGV 256^3 D3Q27: KE worst relative difference vs FP64 %.2e" % ke_err.max())
    assert ke_err.max() < 1e-5
    planes, st = [int(p) for p in ref["planes"]], int(ref["stride"])
    g = m[:, planes][:, :, ::st, ::st]
    res = pu.compare(g, ref["moments"].astype(np.float64))
    for k in range(10):
        print("C2 moment %d: rel L2 %.2e Linf %.2e" % (k, *res[k]))
    bad = per_moment_bounds(res, {k: (0.0, 0.0) for k in res})
    assert not bad, "; ".join(bad)


def test_fp16_batch_members_match_fp64_oracle():
    steps = 500
    specs = [((24, 28, 20), 100.0), ((32, 24, 30), 400.0), ((20, 20, 20), 50.0)]
    b = mrlbm.Batch(mrlbm.D3Q19, mrlbm.F16)
    mem = []
    for (nx, ny, nz), re in specs:
        d = mrlbm.lid_cavity_desc(nx, re=re, lid_u=0.05, storage=mrlbm.F16, ny=ny, nz=nz)
        m = b.add(d)
        nt = mrlbm.lid_cavity_node_types(nx, ny, nz, 1)
        m.set_node_types(nt)
        m.init_uniform()
        mem.append((m, d, nt, pu.gpu_to_oracle_layout(m.moments())))
    b.step(steps)
    b.synchronize()
    errs = []
    for m, d, nt, m0 in mem:
        o = pu.oracle_for(d, nt)
        o.set_moments(m0)
        o.step(steps)
        e = pu.velocity_rel_l2(m.moments(), o.moments())
        errs.append(e)
        print("FP16 batch member %dx%dx%d: u rel L2 vs FP64 %.3e" % (d.nx, d.ny, d.nz, e))
    b.close()
    # 16-bit rounding of the stored moments each step
    assert max(errs) < 5e-3


def test_fp16_served_powerlaw_duct_matches_fp64_oracle():
    steps, n = 400, 32
    req = mrlbm.make_request(mrlbm.REQ_DUCT, n, nnf_n=0.8, solid_fraction=0.05, seed=11)
    d, nt = mrlbm.request_describe(req, mrlbm.F16)
    alone = mrlbm.request_domain(req, mrlbm.F16)
    m0 = pu.gpu_to_oracle_layout(alone.moments())
    alone.close()
    srv = mrlbm.Server(storage=mrlbm.F16, hbm_budget=150e9, max_active=8, steps_per_tick=100,
                       residual_tol=1e-12, max_steps=steps, keep_results=True)
    rid = srv.submit(req)
    while True:
        active = srv.tick()
        if active == 0 and srv.stats()["queued"] == 0:
            break
    res = srv.result(rid)
    g = srv.moments(rid, n, 11)
    srv.close()
    assert res["status"] == 0 and res["steps"] == steps
    o = pu.oracle_for(d, nt)
    o.set_moments(m0)
    o.step(steps)
    om = o.moments()
    fluid = nt != mrlbm.NODE_SOLID
    e = pu.velocity_rel_l2(g, om, fluid)
    ew = pu.compare(g, om, fluid)[10]
    print("FP16 served power-law duct %d^3: u rel L2 vs FP64 %.3e, omega rel L2 %.3e" % (n, e, ew[0]))
    assert e < 2e-2 and ew[0] < 2e-2
