"""C-ABI library on the CPU: it loads, exports every declared symbol, and its
host-side logic (node-type builders, moment-BC matrices) matches the oracle.
No device work is done here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import lattice_np
import oracle_ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    import mrlbm
    return mrlbm


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "mrlbm.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mrlbm_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    mrlbm = _lib()
    L = mrlbm.lib()
    names = declared_symbols()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert b"sm_100a" in L.mrlbm_version()


def test_lid_cavity_typing_matches_reference_rules():
    mrlbm = _lib()
    nx, ny, nz = 10, 9, 8
    t = mrlbm.lid_cavity_node_types(nx, ny, nz, 1)
    F = lattice_np.FACES
    lid = F["NORTH"] | mrlbm.BC_VELOCITY_WALL | mrlbm.BC_VELOCITY_INDEX(1)
    # restatement of src/cases/lidDrivenCavity_3D/bc_initialization.inc
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if y == ny - 1:
                    want = lid
                else:
                    want = 0
                    if y == 0: want |= F["SOUTH"]
                    if x == 0: want |= F["WEST"]
                    if x == nx - 1: want |= F["EAST"]
                    if z == 0: want |= F["BACK"]
                    if z == nz - 1: want |= F["FRONT"]
                assert t[z, y, x] == want, (x, y, z)
    # corner masks equal the reference's named constants
    assert t[0, 0, 0] == 0b01111111           # SOUTH_WEST_BACK
    assert t[nz - 1, 0, nx - 1] == 0b11111011  # SOUTH_EAST_FRONT


def bc_id_restated(solid, x, y, z):
    """Octant marking of src/lbmInitialization.cu:1080-1227 (periodic wrap)."""
    nz, ny, nx = solid.shape
    m = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if not (dx or dy or dz):
                    continue
                if solid[(z + dz) % nz, (y + dy) % ny, (x + dx) % nx]:
                    for o in range(8):
                        s = ((1 if o & 1 else -1), (1 if o & 2 else -1), (1 if o & 4 else -1))
                        if all(d == 0 or d == sv for d, sv in zip((dx, dy, dz), s)):
                            m |= 1 << o
    return m


def test_voxel_typing_matches_bc_id():
    mrlbm = _lib()
    rng = np.random.default_rng(3)
    solid = (rng.random((7, 8, 9)) < 0.15).astype(np.uint8)
    t = mrlbm.voxel_node_types(solid, (1, 1, 1))
    for z in range(7):
        for y in range(8):
            for x in range(9):
                if solid[z, y, x]:
                    assert t[z, y, x] == 0xFF
                else:
                    want = bc_id_restated(solid, x, y, z)
                    assert t[z, y, x] == (0xFE if want == 0xFF else want)


def test_voxel_file_loading_matches_read_xyz_file_and_define_voxel_bc(tmp_path):
    """mrlbm_voxel_mark_csv + mrlbm_voxel_resolve against a restatement of the
    reference's read_xyz_file (src/lbmInitialization.cu:978-1039: solid
    voxels, their 26 neighbours marked MISSING_DEFINITION with every axis
    wrapped, out-of-grid lines skipped) and define_voxel_bc / bc_id (wrapped
    octant masks; a mask of all eight octants is the solid word)."""
    mrlbm = _lib()
    L = mrlbm.lib()
    nx, ny, nz = 9, 8, 7
    rng = np.random.default_rng(11)
    pts = [tuple(int(v) for v in p) for p in rng.integers(0, [nx, ny, nz], size=(25, 3))]
    pts += [(0, 0, 0), (nx - 1, 3, 2), (4, ny - 1, nz - 1), (nx + 3, 1, 1), (2, 2, nz)]   # wrap + out of grid
    csv = tmp_path / "vox.csv"
    csv.write_text("".join("%d,%d,%d\n" % p for p in pts))
    nt = np.zeros((nz, ny, nx), dtype=np.uint32)
    count = C.c_longlong()
    rc = L.mrlbm_voxel_mark_csv(str(csv).encode(), nx, ny, nz, nt.ctypes.data_as(C.POINTER(C.c_uint32)),
                                C.byref(count))
    assert rc == 0
    # restatement of read_xyz_file
    want = np.zeros((nz, ny, nx), dtype=np.int64)
    n_in = 0
    for x, y, z in pts:
        if x >= nx or y >= ny or z >= nz:
            continue
        n_in += 1
        want[z, y, x] = 0xFF
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    k = ((z + dz) % nz, (y + dy) % ny, (x + dx) % nx)
                    if k == (z, y, x) or want[k] == 0xFF:
                        continue
                    want[k] = 0xFFFFFFFF
    assert count.value == n_in
    assert np.array_equal(nt.astype(np.int64), want)
    rc = L.mrlbm_voxel_resolve(nx, ny, nz, nt.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert rc == 0
    solid = (want == 0xFF).astype(np.uint8)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if want[z, y, x] == 0xFFFFFFFF:
                    assert nt[z, y, x] == bc_id_restated(solid, x, y, z), (x, y, z)
                else:
                    assert nt[z, y, x] == want[z, y, x]


def test_voxel_typing_walls_on_nonperiodic_axes():
    mrlbm = _lib()
    solid = np.zeros((6, 5, 4), dtype=np.uint8)
    t = mrlbm.voxel_node_types(solid, (0, 0, 1))
    F = lattice_np.FACES
    assert t[2, 0, 2] == F["SOUTH"]
    assert t[2, 0, 0] == F["SOUTH"] | F["WEST"]
    assert t[2, 2, 3] == F["EAST"]
    assert t[2, 2, 2] == 0


@pytest.mark.parametrize("lattice,mq", [(19, 19), (27, 19), (27, 27)])
def test_bc_matrices_match_oracle(lattice, mq):
    """The Sherman-Morrison form the kernel evaluates equals the oracle's
    direct 7x7 solve, for omegas away from the expansion point."""
    mrlbm = _lib()
    L = oracle_ffi.lib()
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    rng = np.random.default_rng(11)
    omega0 = 1.0 / 0.596
    uvel = [(0, 0, 0), (0.05, 0.0, 0.0), (0.0, 0.01, -0.02), (0, 0, 0)]
    types = list(lattice_np.wall_types().values()) + [0x13, 0x80, 0xC3]
    for t in types:
        for vel in (0, 1, 2):
            word = t | (mrlbm.BC_VELOCITY_WALL | mrlbm.BC_VELOCITY_INDEX(vel) if vel else 0)
            data, known = mrlbm.bc_class_info(lattice, word, uvel, omega0, bc_matrix_q=mq)
            assert known == L.orc_known_mask(lattice, t)
            Ainv = data[:49].reshape(7, 7).astype(np.float64)
            v, qa, s = data[49:56], data[56:63], data[63]
            m = rng.normal(0, 0.05, 10)
            f = np.zeros(lattice)
            L.orc_reconstruct(lattice, 1.0, P(m), P(f))
            f *= 1 + rng.normal(0, 1e-3, lattice)
            kb = np.array([(known >> i) & 1 for i in range(lattice)], dtype=bool)
            fk = np.where(kb, f, 0.0)
            cx, cy, cz = lattice_np.CX[:lattice], lattice_np.CY[:lattice], lattice_np.CZ[:lattice]
            b0 = fk.sum()
            b = np.array([b0, (fk * cx * cx).sum() - b0 / 3, (fk * cx * cy).sum(), (fk * cx * cz).sum(),
                          (fk * cy * cy).sum() - b0 / 3, (fk * cy * cz).sum(), (fk * cz * cz).sum() - b0 / 3])
            u = np.array(uvel[vel] if vel else (0, 0, 0), dtype=np.float64)
            for om in (omega0, 0.9, 1.4, 1.9):
                X = Ainv @ b
                dw = om - omega0
                X = X - v * (dw * (qa @ b) / (1 + dw * s))
                ref = np.zeros(10)
                assert L.orc_bc_solve(lattice, mq, known, P(u), om, P(f), P(ref)) == 0
                np.testing.assert_allclose(X[0], ref[0], rtol=2e-6)
                np.testing.assert_allclose(X[1:] / X[0], ref[4:], rtol=2e-4, atol=2e-7)


def test_thermal_descriptor_rules():
    """The thermal scalar is accepted on D3Q19 with FP32 storage and a
    Newtonian fluid (the reference's thermal cases), with four more stored
    moments; other combinations are rejected before anything is allocated."""
    import mrlbm
    th = dict(diffusivity=0.01, reference=1.0, gravity_beta=(1e-5, 0, 0), wall=(1.5, 0.5))
    n = C.c_size_t()
    d = mrlbm.make_desc(16, 12, 8, lattice=19, thermal=th)
    assert mrlbm.lib().mrlbm_domain_bytes(C.byref(d), C.byref(n)) == 0
    pitch = (16 + 4 + 1 + 7) // 8 * 8
    field = pitch * (12 + 2) * (8 + 2)
    assert n.value == 2 * field * 14 * 4 + field
    bad = [mrlbm.make_desc(16, 12, 8, lattice=27, thermal=th),
           mrlbm.make_desc(16, 12, 8, lattice=19, storage=mrlbm.F16, thermal=th),
           mrlbm.make_desc(16, 12, 8, lattice=19, rheology=mrlbm.POWERLAW, thermal=th),
           mrlbm.make_desc(16, 12, 8, lattice=19, thermal=dict(th, diffusivity=0.0))]
    for d in bad:
        assert mrlbm.lib().mrlbm_domain_bytes(C.byref(d), C.byref(n)) == 1   # MRLBM_EINVAL


def test_descriptor_layout_matches_header():
    """The ctypes mirror of mrlbm_desc has the C header's size and offsets."""
    import subprocess
    import tempfile
    import mrlbm
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = ('#include "mrlbm.h"\n#include <stdio.h>\n#include <stddef.h>\n'
           'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(mrlbm_desc), offsetof(mrlbm_desc, bc_matrix_q),'
           ' offsetof(mrlbm_desc, thermal), offsetof(mrlbm_desc, t_wall)); return 0;}\n')
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "sz.c")
        open(c, "w").write(src)
        exe = os.path.join(tmp, "sz")
        subprocess.check_call(["gcc", "-I", os.path.join(root, "include"), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    D = mrlbm.Desc
    assert vals == [C.sizeof(D), D.bc_matrix_q.offset, D.thermal.offset, D.t_wall.offset]


def test_size_limits():
    """Grids up to 8192 per axis whose padded plane stack of one moment stays
    below 2^32 nodes (the step kernel's 32-bit offsets) are accepted; larger
    ones and empty axes are rejected before anything is allocated."""
    import mrlbm
    n = C.c_size_t()
    ok = mrlbm.make_desc(1600, 1600, 1600, lattice=19, storage=mrlbm.F16)
    assert mrlbm.lib().mrlbm_domain_bytes(C.byref(ok), C.byref(n)) == 0
    for shape in ((2048, 2048, 2048), (0, 8, 8), (8, 8, 8193)):
        d = mrlbm.make_desc(*shape, lattice=19)
        assert mrlbm.lib().mrlbm_domain_bytes(C.byref(d), C.byref(n)) == 1, shape
