"""The FP64 oracle against the reference's own per-node arithmetic.

Golden vectors in tests/golden/ref_kat.npz come from the reference snippets
compiled on the host (tests/golden/make_golden.py); when oracle/_ref is built
the same checks also run live against fresh random inputs.
"""
import ctypes as C
import os

import numpy as np
import pytest

import lattice_np
import oracle_ffi

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_kat.npz"))
P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
L = oracle_ffi.lib()


def orc_recon(q, m):
    f = np.zeros(q)
    L.orc_reconstruct(q, 1.0, P(np.ascontiguousarray(m, dtype=np.float64)), P(f))
    return f


def orc_bc(q, mq, t, u, om, f):
    out = np.zeros(10)
    rc = L.orc_bc_solve(q, mq, L.orc_known_mask(q, int(t)), P(np.asarray(u, dtype=np.float64)), float(om),
                        P(np.ascontiguousarray(f)), P(out))
    assert rc == 0
    return out


@pytest.mark.parametrize("q", [19, 27])
def test_reconstruction_golden(q):
    ins, outs = GOLD["recon%d_in" % q], GOLD["recon%d_out" % q]
    for m, ref in zip(ins, outs):
        np.testing.assert_allclose(orc_recon(q, m), ref, rtol=1e-13, atol=1e-15)


def test_collision_golden():
    for row, ref in zip(GOLD["coll_in"], GOLD["coll_out"]):
        m, rho, F, om = row[:10], row[10], row[11:14], row[14]
        d = oracle_ffi.make_desc(4, 4, 4, force=F)
        mac = np.array([rho, m[1] / 3, m[2] / 3, m[3] / 3, m[4] / 4.5, m[5] / 9, m[6] / 9, m[7] / 4.5, m[8] / 9,
                        m[9] / 4.5])
        out = np.zeros(11)
        L.orc_collide(C.byref(d), P(mac), float(om), P(out), 10)
        np.testing.assert_allclose(out[1:10], ref[1:10], rtol=1e-12, atol=1e-15)


def test_lid_cavity_walls_golden():
    """All 26 face/edge/corner no-slip walls and the moving lid (NORTH)."""
    n = 0
    for t, f, om, umax, ref in zip(GOLD["lid_type"], GOLD["lid_pops"], GOLD["lid_omega"], GOLD["lid_umax"],
                                   GOLD["lid_out"]):
        u = (umax, 0, 0) if t == lattice_np.FACES["NORTH"] else (0, 0, 0)
        np.testing.assert_allclose(orc_bc(19, 19, t, u, om, f), ref, rtol=1e-11, atol=1e-14)
        n += 1
    assert n == 26 * 3


def test_voxel_octant_masks_golden():
    """All 254 octant masks of the voxel BC table."""
    assert len(GOLD["vox_type"]) == 254
    for t, f, om, ref in zip(GOLD["vox_type"], GOLD["vox_pops"], GOLD["vox_omega"], GOLD["vox_out"]):
        np.testing.assert_allclose(orc_bc(19, 19, t, (0, 0, 0), om, f), ref, rtol=1e-11, atol=1e-14)


def test_d3q27_plate_walls_golden():
    """The reference's D3Q27 walls are the D3Q19 closed forms on D3Q27 known sets."""
    for t, f, om, ref in zip(GOLD["pl27_type"], GOLD["pl27_pops"], GOLD["pl27_omega"], GOLD["pl27_out"]):
        np.testing.assert_allclose(orc_bc(27, 19, t, (0, 0, 0), om, f), ref, rtol=1e-11, atol=1e-14)
        # the lattice-consistent D3Q27 system gives a different (documented) answer
        alt = orc_bc(27, 27, t, (0, 0, 0), om, f)
        assert np.max(np.abs(alt - ref)) > 1e-6


def test_known_mask_faces():
    km = lambda t: L.orc_known_mask(19, t)  # noqa: E731
    # south wall (y=0): known populations are those with c_y <= 0
    want = sum(1 << i for i in range(19) if lattice_np.CY[i] <= 0)
    assert km(lattice_np.FACES["SOUTH"]) == want
    assert km(0) == (1 << 19) - 1


def test_live_reference_snippets():
    R = oracle_ffi.ref_kat()
    if R is None:
        pytest.skip("oracle/_ref not built (needs the reference source tree)")
    rng = np.random.default_rng(7)
    for t in range(1, 255):
        f = orc_recon(19, rng.normal(0, 0.05, 10)) * (1 + rng.normal(0, 1e-3, 19))
        om = rng.uniform(0.6, 1.9)
        r = np.zeros(10)
        assert R.ref_bc_voxel_q19(t, P(f), om, 1.0, P(r)) == 1
        np.testing.assert_allclose(orc_bc(19, 19, t, (0, 0, 0), om, f), r, rtol=1e-11, atol=1e-14)


def test_nnf_powerlaw_newtonian_limit():
    # n = 1: a omega + |S|/2 omega - |S| = 0 with a = K |S| / (rho0 cs2) -> omega = 1/tau
    tau = 0.8
    K = (tau - 0.5) / 3
    for s in (1e-4, 1e-3, 1e-2):
        om = L.orc_nnf_powerlaw(1.0, s, 1.0, K, 1.0)
        assert abs(om - 1 / tau) < 1e-9
    assert L.orc_nnf_powerlaw(1.0, 1e-7, 0.7, K, 1.0) == 0.0


def test_nnf_bingham():
    assert L.orc_nnf_bingham(1e-3, 1.2, 2e-3) == 0.0
    assert abs(L.orc_nnf_bingham(4e-3, 1.2, 1e-3) - 1.2 * 0.75) < 1e-15


def test_fp32_build_is_the_same_algorithm_in_fp32():
    """The FP32 build (the round-off yardstick for driven-flow parity) follows
    the FP64 oracle to FP32 accuracy on a short Taylor-Green run, and differs
    from it (it really computes in FP32)."""
    n, u0 = 16, 0.04
    L = n / (2 * np.pi)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ux = u0 * np.sin(x / L) * np.cos(y / L) * np.cos(z / L)
    uy = -u0 * np.cos(x / L) * np.sin(y / L) * np.cos(z / L)
    desc = oracle_ffi.make_desc(n, n, n, q=19, tau=0.6)
    a, b = oracle_ffi.OracleDomain(desc), oracle_ffi.OracleDomain(desc, fp32=True)
    a.init_from_macro(np.ones_like(ux), ux, uy, 0 * ux)
    m0 = a.moments().astype(np.float32).astype(np.float64)
    a.set_moments(m0)
    b.set_moments(m0)
    a.step(20)
    b.step(20)
    ma, mb = a.moments(), b.moments()
    err = np.linalg.norm(mb[..., 1:4] - ma[..., 1:4]) / np.linalg.norm(ma[..., 1:4])
    assert 1e-9 < err < 1e-4, err
    assert np.array_equal(mb, mb.astype(np.float32).astype(np.float64))


def test_thermal_reconstruction_golden():
    """D3G19 populations of the thermal scalar against G_SCALAR/reconstruction.inc.
    The snippet takes the diffusive correction ud directly; the oracle forms it
    as coef (q3 / C - u3), so q3 is chosen to give the same ud."""
    coef = 0.37
    for row, ref in zip(GOLD["g19_in"], GOLD["g19_out"]):
        c, u3, ud3 = row[0], np.ascontiguousarray(row[1:4]), row[4:7]
        q3 = np.ascontiguousarray(c * (u3 + ud3 / coef))
        g = np.zeros(19)
        L.orc_reconstruct_g(coef, float(c), P(u3), P(q3), P(g))
        np.testing.assert_allclose(g, ref, rtol=1e-12, atol=1e-15)


def test_thermal_coefficient_golden():
    """G_DIFF_FLUC_COEF from T_DIFFUSIVITY as the Rayleigh-Benard case computes it."""
    rc = GOLD["rbp_const"]
    assert abs(L.orc_thermal_coef(rc[1]) - rc[0]) < 1e-15
    # T_gravity_t_beta = Ra alpha nu / (dT L^3) with Ra = 1e5, dT = 1, L = N = 64
    assert abs(rc[2] - 1e5 * rc[1] * rc[3] / 64 ** 3) < 1e-18


def test_thermal_sums_recover_moments():
    """Sum g = C and 3 sum g c = C (u3 + coef (q3 / C - u3)): the scalar is
    conserved by the reconstruction and its flux relaxes towards C u."""
    rng = np.random.default_rng(11)
    for _ in range(32):
        c = rng.uniform(0.5, 1.5)
        u3, q3 = rng.normal(0, 0.1, 3), rng.normal(0, 0.1, 3)
        coef = rng.uniform(-0.99, 0.9)
        g, cq = np.zeros(19), np.zeros(4)
        L.orc_reconstruct_g(coef, c, P(u3), P(q3), P(g))
        L.orc_sums_g(P(g), 0.0, P(cq))
        np.testing.assert_allclose(cq[0], c, rtol=1e-14)
        np.testing.assert_allclose(cq[1:], c * (u3 + coef * (q3 / c - u3)), rtol=1e-12, atol=1e-15)


def test_thermal_face_normals():
    side = C.c_int(0)
    for name, axis, sd in (("WEST", 0, -1), ("EAST", 0, 1), ("SOUTH", 1, -1), ("NORTH", 1, 1), ("BACK", 2, -1),
                           ("FRONT", 2, 1)):
        assert L.orc_face_normal(lattice_np.FACES[name], C.byref(side)) == axis
        assert side.value == sd
    # an edge has two solid halves: no single normal
    assert L.orc_face_normal(lattice_np.FACES["WEST"] | lattice_np.FACES["SOUTH"], C.byref(side)) == -1


def test_rayleigh_benard_walls_golden():
    """The thermal Rayleigh-Benard case writes its walls in its own closed
    forms (wall normal l, src/cases/rayleighBenard_Periodic/bc_definition.inc);
    they are the same moment-BC system: faces and edges to round-off."""
    for t, f, om, ref in zip(GOLD["rb_type"], GOLD["rb_pops"], GOLD["rb_omega"], GOLD["rb_out"]):
        np.testing.assert_allclose(orc_bc(19, 19, t, (0, 0, 0), om, f), ref, rtol=1e-11, atol=1e-14)
