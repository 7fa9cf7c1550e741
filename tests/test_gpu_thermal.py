"""Thermal scalar C on D3G19 (the reference's THERMAL_MODEL: SECOND_DIST +
CONVECTION_DIFFUSION_TRANSPORT) through the C ABI, against the FP64 oracle.

Cases follow the reference's thermal cases at small sizes: a periodic box
with a scalar blob carried by a uniform flow (bulk transport, Boussinesq
force); the Rayleigh-Benard cell of src/cases/rayleighBenard_Periodic (hot and
cold walls in x with the neighbour-flux rule, gravity along x, periodic y and
z); a closed cell with Dirichlet side walls and adiabatic (mirrored) top and
bottom, src/cases/rayleighBenard_Closed; and walls that keep their stored
values next to an internal heat source.  Both sides start from the same
stored moments.  FP32 drift is measured against the oracle's FP32 build run
from the same start (the yardstick of test_gpu_parity.py): each moment's
error must stay within twice that build's error or the fixed bound below.
"""
import numpy as np
import pytest

import mrlbm
import parity_util as pu

pytestmark = pytest.mark.gpu

# fixed bounds (relative L2, relative Linf) for flow moments, second moments,
# C and its flux
TOL = {"u": (2e-5, 2e-4), "pi": (3e-4, 2e-3), "c": (2e-6, 2e-5), "q": (1e-4, 1e-3)}


def bound(k):
    if k <= 3:
        return TOL["u"]
    if k <= 9:
        return TOL["pi"]
    return TOL["c"] if k == 10 else TOL["q"]


def thermal_desc(nx, ny, nz, periodic, tau, alpha, gbeta, wall=(1.5, 0.5, 1.0, 1.0), source=0.0):
    return mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=periodic, tau=tau,
                           thermal=dict(diffusivity=alpha, reference=1.0, gravity_beta=gbeta, source=source,
                                        wall=wall))


def run_pair(desc, steps, node_types=None, init=None, fluid=None):
    dom = mrlbm.Domain(desc)
    assert dom.nm == 14
    if node_types is not None:
        dom.set_node_types(node_types)
    dom.init_uniform()
    if init is not None:
        init(dom)
    m0 = pu.gpu_to_oracle_layout(dom.moments())
    orc = pu.oracle_for(desc, node_types)
    orc.set_moments(m0)
    o32 = pu.oracle_for(desc, node_types, fp32=True)
    o32.set_moments(m0)
    dom.step(steps)
    orc.step(steps)
    o32.step(steps)
    g, o = dom.moments(), orc.moments()
    dom.close()
    res = pu.compare(g, o, fluid)
    yard = pu.compare(np.moveaxis(o32.moments(), -1, 0), o, fluid)
    return g, o, res, yard


def assert_close(res, yard):
    for k, (e2, einf) in res.items():
        a2, ainf = bound(k)
        a2, ainf = max(a2, 2 * yard[k][0]), max(ainf, 2 * yard[k][1])
        assert e2 <= a2 and einf <= ainf, "moment %d: rel L2 %.3e (bound %.1e), rel Linf %.3e (bound %.1e)" % (
            k, e2, a2, einf, ainf)


def node_types(nx, ny, nz, x_walls=None, y_walls=None):
    """x_walls / y_walls: (low word bits, high word bits) added to the face
    octant masks of the x = 0 / nx-1 and y = 0 / ny-1 planes; nodes on both
    take the edge mask with the low/high bits of the x walls."""
    t = np.zeros((nz, ny, nx), dtype=np.uint32)
    if y_walls is not None:
        t[:, 0, :] = mrlbm.SOUTH | y_walls[0]
        t[:, -1, :] = mrlbm.NORTH | y_walls[1]
    if x_walls is not None:
        t[:, :, 0] = mrlbm.WEST | x_walls[0]
        t[:, :, -1] = mrlbm.EAST | x_walls[1]
        if y_walls is not None:
            for yi, ym in ((0, mrlbm.SOUTH), (-1, mrlbm.NORTH)):
                t[:, yi, 0] = mrlbm.WEST | ym | x_walls[0]
                t[:, yi, -1] = mrlbm.EAST | ym | x_walls[1]
    return t


def test_thermal_periodic_blob_transport_and_conservation():
    nx, ny, nz = 40, 34, 30   # not multiples of the 30 x 14 column tile
    d = thermal_desc(nx, ny, nz, (1, 1, 1), tau=0.7, alpha=0.02, gbeta=(0.0, 0.0, 2e-5))
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    blob = 1.0 + 0.2 * np.exp(-((x - 20) ** 2 + (y - 17) ** 2 + (z - 15) ** 2) / (2 * 5.0 ** 2))

    def init(dom):
        dom.init_uniform((0.03, -0.02, 0.01))
        m = dom.moments()
        m[10] = blob
        dom.set_moments(m)

    g, o, res, yard = run_pair(d, 60, init=init)
    assert_close(res, yard)
    # the scalar is conserved by the periodic step (no source): FP32 sums
    c0, c1 = float(np.sum(blob.astype(np.float32), dtype=np.float64)), float(np.sum(g[10], dtype=np.float64))
    assert abs(c1 - c0) / c0 < 2e-6
    # and it moved with the flow: the blob's centre of mass advanced by about u t
    w = g[10].astype(np.float64) - 1.0
    cx = float(np.sum(w * x) / np.sum(w))
    assert 20.8 < cx < 22.6   # 20 + 0.03 * 60 = 21.8


def test_rayleigh_benard_periodic_cell():
    """src/cases/rayleighBenard_Periodic at 32 x 24 x 6: hot WEST / cold EAST
    walls with the neighbour-flux rule, gravity along x, Pr = 10, Ra = 1e5."""
    nx, ny, nz = 32, 24, 6
    tau = 0.55
    nu = (tau - 0.5) / 3
    alpha = nu / 10.0
    gb = 1e5 * alpha * nu / (1.0 * nx ** 3)
    d = thermal_desc(nx, ny, nz, (0, 1, 1), tau=tau, alpha=alpha, gbeta=(gb, 0.0, 0.0), wall=(1.5, 0.5, 1.0, 1.0))
    rule = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET_FLUX)
    nt = node_types(nx, ny, nz, x_walls=(rule | mrlbm.THERMAL_INDEX(0), rule | mrlbm.THERMAL_INDEX(1)))
    g, o, res, yard = run_pair(d, 200, node_types=nt)
    assert_close(res, yard)
    # the walls hold their temperatures and heat has entered the cell
    assert np.allclose(g[10][:, :, 0], 1.5) and np.allclose(g[10][:, :, -1], 0.5)
    assert float(np.mean(g[10][:, :, 1])) > 1.0 > float(np.mean(g[10][:, :, -2]))


def test_closed_cell_adiabatic_walls():
    """src/cases/rayleighBenard_Closed: Dirichlet side walls in x (edges too),
    adiabatic mirrored walls in y, periodic z; gravity along y."""
    nx, ny, nz = 28, 26, 8
    tau = 0.6
    nu = (tau - 0.5) / 3
    alpha = nu / 0.71
    gb = 1e4 * alpha * nu / (1.0 * ny ** 3)
    d = thermal_desc(nx, ny, nz, (0, 0, 1), tau=tau, alpha=alpha, gbeta=(0.0, gb, 0.0), wall=(1.5, 0.5, 1.0, 1.0))
    dr = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET)
    ad = mrlbm.THERMAL_RULE(mrlbm.THERMAL_ADIABATIC)
    nt = node_types(nx, ny, nz, x_walls=(dr | mrlbm.THERMAL_INDEX(0), dr | mrlbm.THERMAL_INDEX(1)),
                    y_walls=(ad, ad))
    g, o, res, yard = run_pair(d, 150, node_types=nt)
    assert_close(res, yard)


def test_keep_rule_walls_and_internal_source():
    """Walls without a thermal rule keep their stored C and flux; bulk nodes
    gain the internal source every step (T_Q_INTERNAL_D_Cp)."""
    nx, ny, nz = 24, 20, 12
    d = thermal_desc(nx, ny, nz, (1, 0, 1), tau=0.8, alpha=0.05, gbeta=(0.0, 1e-5, 0.0), source=1e-4)
    nt = node_types(nx, ny, nz, y_walls=(0, 0))

    def init(dom):
        m = dom.moments()
        m[10][:, 0, :] = 0.8
        m[10][:, -1, :] = 1.2
        dom.set_moments(m)

    g, o, res, yard = run_pair(d, 80, node_types=nt, init=init)
    assert_close(res, yard)
    assert np.all(g[10][:, 0, :] == np.float32(0.8)) and np.all(g[10][:, -1, :] == np.float32(1.2))


def test_flux_rule_needs_a_face_node():
    d = thermal_desc(8, 8, 8, (0, 0, 1), tau=0.8, alpha=0.05, gbeta=(0.0, 0.0, 0.0))
    dom = mrlbm.Domain(d)
    t = np.zeros((8, 8, 8), dtype=np.uint32)
    t[:, 0, 0] = mrlbm.WEST | mrlbm.SOUTH | mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET_FLUX)
    with pytest.raises(mrlbm.MrlbmError):
        dom.set_node_types(t)
    dom.close()


def test_thermal_files():
    """The scalar goes to <id>_C<step>.bin and to the VTK file's SCALARS C,
    as the reference writes it with SECOND_DIST (src/saveData.cu:192-230, 371-376)."""
    import os
    import tempfile
    d = thermal_desc(16, 8, 8, (1, 1, 1), tau=0.8, alpha=0.05, gbeta=(0.0, 0.0, 0.0))
    dom = mrlbm.Domain(d)
    dom.init_uniform()
    m = dom.moments()
    m[10] = 1.0 + 0.01 * np.arange(m[10].size, dtype=np.float32).reshape(m[10].shape) / m[10].size
    dom.set_moments(m)
    with tempfile.TemporaryDirectory() as tmp:
        dom.save_macr_bin(tmp, "th", 7)
        c = np.fromfile(os.path.join(tmp, "th", "th_C000007.bin"), dtype=np.float32)
        assert np.array_equal(c, m[10].reshape(-1))
        dom.save_vtk(tmp, "th", 7)
        raw = open(os.path.join(tmp, "th", "th_vtk000007.vtk"), "rb").read()
        at = raw.index(b"SCALARS C float 1\nLOOKUP_TABLE default\n") + len(b"SCALARS C float 1\nLOOKUP_TABLE default\n")
        cv = np.frombuffer(raw[at:at + 4 * c.size], dtype=">f4")
        assert np.array_equal(cv.astype(np.float32), m[10].reshape(-1))
    dom.close()


def test_thermal_checkpoint_round_trip():
    """Checkpoints carry the four thermal moments in _fMom.bin and the D3G19
    ghost faces in _g_fGhost.{X,Y,Z}_{0,1}.bin (src/checkpoint.cu:188-194:
    5 populations per node of every 8^3 block's face, n^3 / 8 nodes per
    orientation, src/definitions.h:113-115)."""
    import os
    import tempfile
    n = 16
    d = thermal_desc(n, n, n, (1, 1, 1), tau=0.8, alpha=0.05, gbeta=(0.0, 0.0, 1e-5))
    a = mrlbm.Domain(d)
    a.init_uniform((0.01, 0.0, 0.0))
    m = a.moments()
    m[10] = 1.0 + 0.1 * np.random.default_rng(3).random(m[10].shape, dtype=np.float32)
    a.set_moments(m)
    a.step(5)
    with tempfile.TemporaryDirectory() as tmp:
        a.save_checkpoint(tmp, "th", 5)
        for f in ("X_0", "X_1", "Y_0", "Y_1", "Z_0", "Z_1"):
            assert os.path.getsize(os.path.join(tmp, "th", "checkpoint", "_g_fGhost.%s.bin" % f)) == 4 * 5 * n ** 3 // 8
        b = mrlbm.Domain(d)
        assert b.load_checkpoint(tmp, "th") == 6
        assert np.array_equal(a.moments(), b.moments())
        a.step(3)
        b.step(3)
        assert np.array_equal(a.moments(), b.moments())
        b.close()
    a.close()


def test_rayleigh_benard_matches_reference_program(tmp_path):
    """The reference's own CUDA program for rayleighBenard_Periodic (built for
    sm_100 by oracle/build_ref_cuda.sh: 64 x 64 x 8, D3Q19 + D3G19, Pr 10,
    Ra 1e5, hot WEST / cold EAST, gravity along x, 1000 steps) against this
    library set up from the same constants, both against the FP64 oracle.
    The case's wall closed forms are the library's moment-BC system
    (tests/test_oracle_kat.py), and its neighbour-flux wall rule reads a value
    that no thread of the step has rewritten yet, so both sides compute the
    same arithmetic up to FP32 operation order.

    With gravity normal to the walls and no perturbation the cell conducts:
    the exact velocity is zero and what the solvers carry (|u| ~ 1e-6) is
    FP32 round-off of the momentum sums, so velocities are compared in
    absolute terms, against the case's free-fall velocity sqrt(g beta dT L)."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "refsim_rb64")
    if not os.path.exists(exe):
        pytest.skip("reference CUDA build missing (oracle/build_ref_cuda.sh needs the reference tree)")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Kernel launch failed" not in r.stdout, r.stdout[-2000:]
    nx, ny, nz, steps = 64, 64, 8, 1000
    ref = {v: np.fromfile(str(tmp_path / "TEST" / "000" / ("000_%s%06d.bin" % (v, steps))), dtype=np.float32)
           .reshape(nz, ny, nx).astype(np.float64) for v in ("rho", "ux", "uy", "uz", "C")}
    # the case's constants (golden copy of rayleighBenard_Periodic/constants.inc)
    const = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kat.npz"))["rbp_const"]
    coef, alpha, gtb, visc, tref, thot, tcold = const[:7]
    d = thermal_desc(nx, ny, nz, (0, 1, 1), tau=0.5 + 3 * visc, alpha=alpha, gbeta=tuple(gtb * const[7:10]),
                     wall=(thot, tcold, tref, tref))
    rule = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET_FLUX)
    nt = node_types(nx, ny, nz, x_walls=(rule | mrlbm.THERMAL_INDEX(0), rule | mrlbm.THERMAL_INDEX(1)))
    dom = mrlbm.Domain(d)
    dom.set_node_types(nt)
    dom.init_uniform()
    orc = pu.oracle_for(d, nt)
    orc.set_moments(pu.gpu_to_oracle_layout(dom.moments()))
    dom.step(steps)
    orc.step(steps)
    g = dom.moments().astype(np.float64)
    o = np.moveaxis(orc.moments(), -1, 0)
    dom.close()
    ours = {"rho": 1.0 + g[0], "ux": g[1], "uy": g[2], "uz": g[3], "C": g[10]}
    fp64 = {"rho": 1.0 + o[0], "ux": o[1], "uy": o[2], "uz": o[3], "C": o[10]}
    u_scale = 3.0 * np.sqrt(gtb * (thot - tcold) * nx)   # stored 3u of the free-fall velocity

    def c_err(a, b):
        return float(np.sqrt(np.sum((a["C"] - b["C"]) ** 2) / np.sum((b["C"] - tref) ** 2)))

    def u_err(a, b):
        return max(float(np.max(np.abs(a[k] - b[k]))) for k in ("ux", "uy", "uz")) / u_scale

    def rho_err(a, b):
        return float(np.max(np.abs(a["rho"] - b["rho"])))

    pairs = {"ours-ref": (ours, ref), "ours-fp64": (ours, fp64), "ref-fp64": (ref, fp64)}
    res = {k: (c_err(*v), u_err(*v), rho_err(*v)) for k, v in pairs.items()}
    for k, (ce, ue, re_) in res.items():
        print("RB 64x64x8 %-9s C rel L2 %.3e, max|du| / U %.3e, max|drho| %.3e" % (k, ce, ue, re_))
    assert res["ours-ref"][0] < 1e-4 and res["ours-ref"][1] < 2e-4 and res["ours-ref"][2] < 1e-5
    # no further from FP64 than the reference program itself (or FP32 level)
    assert res["ours-fp64"][0] <= max(1e-5, 2 * res["ref-fp64"][0])
    assert res["ours-fp64"][1] <= max(1e-5, 2 * res["ref-fp64"][1])
