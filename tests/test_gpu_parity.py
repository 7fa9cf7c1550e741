"""CUDA fused step vs the FP64 oracle, through the C ABI (libmrlbm.so).

Errors are per moment, relative to the norm of the moment's group (rho-rho0
against rho, u components against |u|, second moments against the second
moment group; see parity_util.GROUPS).  Tolerances for FP32 storage and
arithmetic against FP64, after the stated number of steps:
  rho and u: relative L2 <= 2e-5, relative Linf <= 2e-4;
  second moments: relative L2 <= 3e-4, relative Linf <= 2e-3 (they are formed
  as sum(f c c)/rho - 1/3 with |Pi| ~ u^2, so FP32 cancellation against 1/3
  sets their floor, in the reference as here).
Both sides start from the same stored moments (the GPU's own initial state
copied into the oracle), so the comparison isolates the step.

Driven flows (a body force from rest, non-Newtonian omega) accumulate FP32
round-off over the run instead of damping it, so a fixed bound does not fit
them.  Their yardstick is the oracle's own FP32 build (oracle/liboracle_f32.so:
the same restatement in FP32 arithmetic and storage) run from the same start:
the GPU's error against FP64 must stay within twice that build's error (or the
fixed bound, whichever is larger), i.e. no worse than a plain FP32
implementation of the algorithm.
"""
import numpy as np
import pytest

import lattice_np
import mrlbm
import parity_util as pu

pytestmark = pytest.mark.gpu

TOL_L2, TOL_LINF = 2e-5, 2e-4
TOL2_L2, TOL2_LINF = 3e-4, 2e-3   # second moments


def run_pair(desc, steps, node_types=None, init=None, fluid=None, yardstick=False):
    """GPU and FP64 oracle from the same stored start; with yardstick=True also
    the FP32 oracle build, returned as a fourth item (its errors vs FP64)."""
    dom = mrlbm.Domain(desc)
    if node_types is not None:
        dom.set_node_types(node_types)
    if init is None:
        dom.init_uniform()
    else:
        init(dom)
    m0 = pu.gpu_to_oracle_layout(dom.moments())
    orc = pu.oracle_for(desc, node_types)
    orc.set_moments(m0)
    dom.step(steps)
    orc.step(steps)
    g = dom.moments()
    o = orc.moments()
    dom.close()
    if not yardstick:
        return g, o, pu.compare(g, o, fluid)
    o32 = pu.oracle_for(desc, node_types, fp32=True)
    o32.set_moments(m0)
    o32.step(steps)
    y = pu.compare(np.moveaxis(o32.moments(), -1, 0), o, fluid)
    return g, o, pu.compare(g, o, fluid), y


def assert_close(res, l2=TOL_L2, linf=TOL_LINF, l2_2=TOL2_L2, linf_2=TOL2_LINF, skip=(), yard=None):
    for k, (e2, einf) in res.items():
        if k in skip:
            continue
        a2, ainf = (l2_2, linf_2) if 4 <= k <= 9 else (l2, linf)
        if yard is not None:
            a2, ainf = max(a2, 2 * yard[k][0]), max(ainf, 2 * yard[k][1])
        assert e2 <= a2 and einf <= ainf, "moment %d: rel L2 %.3e (bound %.1e), rel Linf %.3e (bound %.1e)" % (
            k, e2, a2, einf, ainf)


def tg_init(u0, L):
    return lambda dom: dom.init_taylor_green(u0, L)


@pytest.mark.parametrize("lattice", [19, 27])
def test_taylor_green_periodic(lattice):
    n = 32
    d = mrlbm.make_desc(n, n, n, lattice=lattice, tau=0.55)
    g, o, res = run_pair(d, 40, init=tg_init(0.04, n / (2 * np.pi)))
    assert_close(res)


def test_random_field_partial_tiles():
    """Sizes that are not multiples of the 30 x 14 x LZ tile, random initial field."""
    nx, ny, nz = 37, 29, 23
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, tau=0.7)
    rng = np.random.default_rng(5)
    rho = 1 + 0.01 * rng.standard_normal((nz, ny, nx))
    u = 0.02 * rng.standard_normal((3, nz, ny, nx))
    g, o, res = run_pair(d, 25, init=lambda dom: dom.init_flow(rho, u[0], u[1], u[2]))
    assert_close(res)


@pytest.mark.parametrize("lattice", [19, 27])
def test_lid_cavity(lattice):
    nx, ny, nz = 24, 20, 16
    d = mrlbm.lid_cavity_desc(nx, re=100.0, lid_u=0.05, lattice=lattice, ny=ny, nz=nz)
    nt = mrlbm.lid_cavity_node_types(nx, ny, nz, 1)
    g, o, res = run_pair(d, 300, node_types=nt)
    assert_close(res, l2=5e-5, linf=5e-4)


def test_duct_voxels_force_newtonian():
    nx, ny, nz = 20, 18, 24
    rng = np.random.default_rng(9)
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    solid[:, 1:-1, 1:-1] = rng.random((nz, ny - 2, nx - 2)) < 0.05
    nt = mrlbm.voxel_node_types(solid, (0, 0, 1))
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(0, 0, 1), tau=0.8, force=(0, 0, 2e-5))
    # from rest |u| grows from zero, so u carries the round-off of rho ~ 1 at
    # a tiny magnitude from the first step on: the FP32 yardstick bounds both
    # an early and a later state
    for steps in (10, 150):
        g, o, res, yard = run_pair(d, steps, node_types=nt, fluid=solid == 0, yardstick=True)
        assert_close(res, yard=yard)


def sheared_start(nx, ny, nz, gamma=2e-3):
    """u_x = gamma (y - ny/2) plus a z wave: |S| is far from the power-law
    cut-off (1e-6) and from a Bingham yield stress of 1e-5 everywhere."""
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ux = gamma * (y - ny / 2) + 0.01 * np.sin(2 * np.pi * z / nz)
    uy = 0.005 * np.sin(2 * np.pi * x / nx)
    uz = 0.005 * np.cos(2 * np.pi * y / ny)
    return lambda dom: dom.init_flow(np.ones_like(ux), ux, uy, uz)


@pytest.mark.parametrize("rheology,kw", [(mrlbm.POWERLAW, dict(nnf_n=0.7)), (mrlbm.POWERLAW, dict(nnf_n=1.15)),
                                         (mrlbm.BINGHAM, dict(nnf_yield=1e-5))])
def test_nonnewtonian_sheared(rheology, kw):
    """Power law and Bingham away from their switching points: FP32 tolerances."""
    nx, ny, nz = 22, 20, 18
    rng = np.random.default_rng(4)
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    solid[:, 2:-2, 2:-2] = rng.random((nz, ny - 4, nx - 4)) < 0.03
    nt = mrlbm.voxel_node_types(solid, (1, 0, 1))
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(1, 0, 1), tau=0.8, force=(3e-6, 0, 1e-6),
                        rheology=rheology, **kw)
    g, o, res, yard = run_pair(d, 60, node_types=nt, init=sheared_start(nx, ny, nz), fluid=solid == 0,
                               yardstick=True)
    assert_close(res, l2=1e-4, linf=2e-3, l2_2=1e-3, linf_2=1e-2, yard=yard)


def test_duct_voxels_force_powerlaw():
    nx, ny, nz = 20, 18, 24
    rng = np.random.default_rng(9)
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    solid[:, 1:-1, 1:-1] = rng.random((nz, ny - 2, nx - 2)) < 0.05
    nt = mrlbm.voxel_node_types(solid, (0, 0, 1))
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(0, 0, 1), tau=0.8, force=(0, 0, 2e-5),
                        rheology=mrlbm.POWERLAW, nnf_n=0.8)
    g, o, res, yard = run_pair(d, 150, node_types=nt, fluid=solid == 0, yardstick=True)
    # the power law sets omega = 0 below |S| = 1e-6 (src/nnf.h:73-74): nodes
    # whose shear crosses that threshold at a different step in FP32 and FP64
    # differ by O(1) in omega, so the bound is looser than for Newtonian flow
    assert_close(res, l2=3e-3, linf=2e-2, l2_2=3e-3, linf_2=2e-2, yard=yard)


def test_bingham_plates():
    nx, ny, nz = 16, 22, 16
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    nt = mrlbm.voxel_node_types(solid, (1, 0, 1))
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(1, 0, 1), tau=0.9, force=(5e-5, 0, 0),
                        rheology=mrlbm.BINGHAM, nnf_yield=1e-5)
    g, o, res, yard = run_pair(d, 150, node_types=nt, yardstick=True)
    # Bingham: omega = omega_p max(0, 1 - S_Y/|S|) switches at the yield
    # surface; FP32 and FP64 place it one node apart in places
    assert_close(res, l2=5e-3, linf=3e-2, l2_2=5e-3, linf_2=3e-2, yard=yard)


@pytest.mark.parametrize("storage,tol", [(mrlbm.F16, 5e-3), (mrlbm.BF16, 4e-2)])
def test_half_storage_taylor_green(storage, tol):
    """16-bit storage, FP32 arithmetic: velocity error vs FP64 stays bounded."""
    n = 32
    d = mrlbm.make_desc(n, n, n, lattice=27, storage=storage, tau=0.55)
    g, o, res = run_pair(d, 40, init=tg_init(0.04, n / (2 * np.pi)))
    err = pu.velocity_rel_l2(g, o)
    assert err < tol, err


def test_graph_equals_eager():
    n = 24
    d = mrlbm.make_desc(n, n, n, lattice=19, tau=0.6)
    a = mrlbm.Domain(d)
    b = mrlbm.Domain(d)
    for dom in (a, b):
        dom.init_taylor_green(0.05, n / (2 * np.pi))
    a.step(37)
    b.step_graph(37)
    assert b.step_count == 37
    np.testing.assert_array_equal(a.moments(), b.moments())


def test_reference_layout_roundtrip():
    nx, ny, nz = 16, 24, 8
    d = mrlbm.make_desc(nx, ny, nz, lattice=19)
    dom = mrlbm.Domain(d)
    rng = np.random.default_rng(1)
    m = rng.standard_normal((10, nz, ny, nx)).astype(np.float32) * 0.01
    dom.set_moments(m)
    ref = dom.moments_ref_layout()
    # idxMom = tx + 8(ty + 8(tz + 8(mom + NM(bx + NBX(by + NBY bz)))))
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    for k in range(10):
        idx = (x % 8) + 8 * ((y % 8) + 8 * ((z % 8) + 8 * (k + 10 * ((x // 8) + (nx // 8) * ((y // 8) + (ny // 8) * (z // 8))))))
        np.testing.assert_array_equal(ref[idx], m[k])
    dom.set_moments_ref_layout(ref)
    np.testing.assert_array_equal(dom.moments(), m)


def test_fp64_reductions():
    n = 24
    d = mrlbm.make_desc(n, n, n, lattice=19)
    dom = mrlbm.Domain(d)
    dom.init_taylor_green(0.05, n / (2 * np.pi))
    dom.step(5)
    m = dom.moments().astype(np.float64)
    s = dom.sums()
    rho = 1.0 + m[0]
    u = m[1:4] / 3.0
    np.testing.assert_allclose(s["mass"], rho.sum(), rtol=1e-12)
    np.testing.assert_allclose(s["kinetic_energy"], 0.5 * (rho * (u ** 2).sum(0)).sum(), rtol=1e-12)
    np.testing.assert_allclose(s["momentum"], (rho * u).reshape(3, -1).sum(1), atol=1e-9)
    assert s["fluid_nodes"] == n ** 3 and s["nonfinite"] == 0
    r0 = dom.residual()
    dom.step(3)
    r1 = dom.residual()
    assert r0 == 1.0 and 0 < r1 < 1


def test_kinetic_energy_decay_matches_oracle():
    """The reference's TGV report (src/cases/taylorGreen/treat_data.inc)."""
    n = 32
    d = mrlbm.make_desc(n, n, n, lattice=27, tau=0.52)
    dom = mrlbm.Domain(d)
    dom.init_taylor_green(0.04, n / (2 * np.pi))
    orc = pu.oracle_for(d)
    orc.set_moments(pu.gpu_to_oracle_layout(dom.moments()))
    for _ in range(4):
        dom.step(25)
        orc.step(25)
        np.testing.assert_allclose(dom.sums()["kinetic_energy"], orc.sums()[4], rtol=1e-5)


def read_vtk(path):
    """Legacy binary VTK structured points: header lines, then big-endian
    float sections (the reference's saveVarVTK layout)."""
    raw = open(path, "rb").read()
    out, pos, n = {}, 0, None
    header = {}
    while pos < len(raw):
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode()
        pos = end + 1
        parts = line.split()
        if not parts:
            continue
        if parts[0] in ("DIMENSIONS", "ORIGIN", "SPACING", "DATASET"):
            header[parts[0]] = parts[1:]
        elif parts[0] == "POINT_DATA":
            n = int(parts[1])
        elif parts[0] == "SCALARS":
            end = raw.index(b"\n", pos)  # LOOKUP_TABLE default
            pos = end + 1
            out[parts[1]] = np.frombuffer(raw, dtype=">f4", count=n, offset=pos)
            pos += 4 * n
        elif parts[0] == "VECTORS":
            out[parts[1]] = np.frombuffer(raw, dtype=">f4", count=3 * n, offset=pos).reshape(n, 3)
            pos += 12 * n
    return header, out


def test_vtk_writer(tmp_path):
    nx, ny, nz = 24, 16, 8
    d = mrlbm.make_desc(nx, ny, nz, lattice=19, tau=0.7, rheology=mrlbm.BINGHAM, nnf_yield=1e-6,
                        periodic=(1, 0, 1), force=(1e-5, 0, 0))
    dom = mrlbm.Domain(d)
    dom.set_node_types(mrlbm.voxel_node_types(np.zeros((nz, ny, nx), np.uint8), (1, 0, 1)))
    dom.init_uniform()
    dom.step(20)
    dom.save_vtk(str(tmp_path), "000", 20)
    m = dom.moments()
    dom.close()
    header, f = read_vtk(tmp_path / "000" / "000_vtk000020.vtk")
    assert header["DIMENSIONS"] == [str(nx), str(ny), str(nz)] and header["DATASET"] == ["STRUCTURED_POINTS"]
    np.testing.assert_array_equal(f["rho"], (np.float32(1.0) + m[0]).reshape(-1))
    np.testing.assert_allclose(f["velocity"], (m[1:4] / np.float32(3.0)).reshape(3, -1).T, rtol=1e-6)
    np.testing.assert_array_equal(f["omega"], m[10].reshape(-1))


def channel_node_types(nx, ny, nz, inlet_index=0):
    """Walled channel along z: no-slip walls on the x and y faces (edges and
    corners with the z faces are walls too), a velocity inlet on the interior
    of z = 0 (BACK + BC_VELOCITY_WALL) and an outflow on the interior of
    z = nz-1 (FRONT + BC_OUTFLOW), as the reference's mountedCube and
    externalFlow cases type them."""
    F = lattice_np.FACES
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    side = (x == 0) | (x == nx - 1) | (y == 0) | (y == ny - 1)
    m = (np.where(x == 0, F["WEST"], 0) | np.where(x == nx - 1, F["EAST"], 0) | np.where(y == 0, F["SOUTH"], 0) |
         np.where(y == ny - 1, F["NORTH"], 0) | np.where(side & (z == 0), F["BACK"], 0) |
         np.where(side & (z == nz - 1), F["FRONT"], 0)).astype(np.uint32)
    m[0][~side[0]] = F["BACK"] | mrlbm.BC_VELOCITY_WALL | mrlbm.BC_VELOCITY_INDEX(inlet_index)
    m[-1][~side[-1]] = F["FRONT"] | mrlbm.BC_OUTFLOW
    return m


@pytest.mark.parametrize("lattice", [19, 27])
def test_channel_velocity_inlet_outflow(lattice):
    """Outflow walls take the moments their inward neighbour stored in the
    previous step (src/cases/mountedCube/bc_definition.inc:18-33) and collide
    them; the channel is driven by a velocity inlet, 250 steps."""
    nx, ny, nz = 20, 18, 36
    nt = channel_node_types(nx, ny, nz)
    d = mrlbm.make_desc(nx, ny, nz, lattice=lattice, periodic=(0, 0, 0), tau=0.7, bc_velocity=[(0.0, 0.0, 0.03)])
    g, o, res, yard = run_pair(d, 250, node_types=nt, yardstick=True)
    assert_close(res, yard=yard)
    # the outlet carries the flow out: its velocity follows the plane before it
    uz = g[3]
    assert float(np.mean(uz[-1, 1:-1, 1:-1])) > 0.0
    assert np.allclose(uz[-1, 1:-1, 1:-1], uz[-2, 1:-1, 1:-1], rtol=0.1, atol=3e-3)


@pytest.mark.parametrize("storage,tol", [(mrlbm.F16, 3e-3), (mrlbm.BF16, 3e-2)])
def test_channel_outflow_half_storage(storage, tol):
    """The outflow read of the 16-bit stored forms (scaled back on load)
    against FP32 storage: relative L2 of u after 150 steps."""
    nx, ny, nz = 20, 18, 36
    nt = channel_node_types(nx, ny, nz)
    out = []
    for st in (mrlbm.F32, storage):
        d = mrlbm.make_desc(nx, ny, nz, lattice=19, storage=st, periodic=(0, 0, 0), tau=0.7,
                            bc_velocity=[(0.0, 0.0, 0.03)])
        dom = mrlbm.Domain(d)
        dom.set_node_types(nt)
        dom.init_uniform()
        dom.step(150)
        out.append(dom.moments()[1:4].astype(np.float64))
        dom.close()
    err = float(np.sqrt(np.sum((out[1] - out[0]) ** 2) / np.sum(out[0] ** 2)))
    assert err < tol, "storage %d: u rel L2 vs FP32 %.3e" % (storage, err)


def test_outflow_needs_a_face_node():
    d = mrlbm.make_desc(8, 8, 8, lattice=19, periodic=(0, 0, 0), tau=0.8)
    dom = mrlbm.Domain(d)
    t = np.zeros((8, 8, 8), dtype=np.uint32)
    t[-1, 0, 0] = lattice_np.FACES["FRONT"] | lattice_np.FACES["WEST"] | mrlbm.BC_OUTFLOW
    with pytest.raises(mrlbm.MrlbmError):
        dom.set_node_types(t)
    dom.close()


def test_batch_rejects_outflow_members():
    b = mrlbm.Batch(mrlbm.D3Q19, mrlbm.F32)
    m = b.add(mrlbm.make_desc(20, 18, 36, lattice=19, periodic=(0, 0, 0), tau=0.7, bc_velocity=[(0, 0, 0.03)]))
    m.set_node_types(channel_node_types(20, 18, 36))
    m.init_uniform()
    with pytest.raises(mrlbm.MrlbmError):
        b.step(1)
    b.close()


def test_bounded_wait_gives_up_and_context_survives():
    """Failure detection without a fault: a device wait on a barrier nothing
    completes gives up after its poll limit and raises the error flag the
    step kernels raise (MRLBM_ETIMEDOUT on the host); the context then runs
    a normal step.  2^16 polls: well under a second."""
    st, sec = mrlbm.selftest_bounded_wait(1 << 16)
    assert st == 6, "expected MRLBM_ETIMEDOUT, got %d" % st   # MRLBM_ETIMEDOUT
    assert 0.0 < sec < 5.0
    d = mrlbm.make_desc(24, 20, 16, lattice=19, tau=0.7)
    g, o, res = run_pair(d, 5, init=tg_init(0.02, 24 / (2 * np.pi)))
    assert_close(res)


@pytest.mark.parametrize("shape,lattice", [((1, 12, 10), 19), ((9, 1, 7), 19), ((8, 6, 1), 27), ((30, 14, 5), 19),
                                           ((31, 15, 3), 27), ((61, 29, 2), 19), ((2, 2, 2), 27)])
def test_edge_shapes_random_field(shape, lattice):
    """Shapes at the edges of the decomposition: one-node axes (a node is its
    own periodic neighbour and holds both ghost copies), columns exactly one
    tile wide and one node over, z depths below the chunk, a 2^3 box; seeded
    random field, periodic, against the oracle."""
    nx, ny, nz = shape
    d = mrlbm.make_desc(nx, ny, nz, lattice=lattice, tau=0.7)
    rng = np.random.default_rng(nx * 10000 + ny * 100 + nz)
    rho = 1 + 0.01 * rng.standard_normal((nz, ny, nx))
    u = 0.02 * rng.standard_normal((3, nz, ny, nx))
    g, o, res = run_pair(d, 12, init=lambda dom: dom.init_flow(rho, u[0], u[1], u[2]))
    assert_close(res)
