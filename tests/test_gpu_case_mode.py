"""Case mode: reference case folders compiled unchanged into this library's
kernels (mr-lbm_b200/casebuild.py; the programs are built into oracle/_ref/cases
by oracle/build_ref_cuda.sh), run next to the reference's own programs on the
same inputs.

* benchmark (README table case, D3Q19 256^3, cuRAND-perturbed field, 1000
  steps): both programs draw the same cuRAND numbers, so their final fields
  must agree to FP32 operation-order level.
* taylorGreen switched to D3Q27, 256^3, Re 1600, u0 0.04, 1000 steps: the
  kinetic-energy reports (every 100 steps) must agree.
* lidDrivenCavity_3D 64^3: the case's own bc_definition.inc running inside the
  z-march kernel must agree with the library's generic moment-BC solver.
* parallelPlates_D3Q19_turbulent_Bingham at 32 x 32 x 64, Re 10, 1000 steps:
  the Bingham fields, and the turbulence statistics its treat_data.inc
  writes through the reference's host context, must agree.
* voxel (an obstacle case whose VOXEL_FILENAME names a CSV of solid nodes),
  64^3, 500 steps, with a sphere and a blob that wraps across the periodic
  faces: the case's voxel file, its 254-mask bc_definition.inc and the
  reference program's own run must agree to FP32 operation order.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import lattice_np
import mrlbm

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def run(exe, workdir):
    if not os.path.exists(exe):
        pytest.skip("%s not built (oracle/build_ref_cuda.sh needs the reference tree)" % exe)
    os.makedirs(workdir, exist_ok=True)
    r = subprocess.run([exe], cwd=workdir, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    m = re.search(r"MLUPS:\s*([0-9.]+)", r.stdout)
    return float(m.group(1)) if m else None


def fields(workdir, n, step):
    base = os.path.join(workdir, "TEST", "000", "000_")
    return {v: np.fromfile(base + "%s%06d.bin" % (v, step), dtype=np.float32).reshape(n, n, n)
            for v in ("rho", "ux", "uy", "uz")}


def u_err(a, b):
    ua = np.stack([a["ux"], a["uy"], a["uz"]])
    ub = np.stack([b["ux"], b["uy"], b["uz"]])
    return lattice_np.rel_l2(ua, ub)


def test_benchmark_case_matches_reference_program(tmp_path):
    """The case's initial velocity is white noise of standard deviation
    0.01 * 0.5 per component (flow_initialization.inc, CURAND_STD_DEV), which
    by step 1000 has decayed by about three orders of magnitude; what is left
    is compared against the initial amplitude, since the relative error of
    the decayed remainder measures FP32 round-off, not the method."""
    ml_ref = run(os.path.join(REF, "refsim_bench256"), tmp_path / "ref")
    ml_ours = run(os.path.join(REF, "cases", "bench256"), tmp_path / "ours")
    a, b = fields(tmp_path / "ours", 256, 1000), fields(tmp_path / "ref", 256, 1000)
    e = u_err(a, b)
    du = np.stack([a[v] - b[v] for v in ("ux", "uy", "uz")])
    # the saved u is the stored 3u (saveData.cu:62-74)
    du_rms = float(np.sqrt(np.mean(du.astype(np.float64) ** 2))) / 3.0
    u_rms = float(np.sqrt(np.mean(np.stack([b[v] for v in ("ux", "uy", "uz")]).astype(np.float64) ** 2))) / 3.0
    drho = float(np.max(np.abs(a["rho"] - b["rho"])))
    print("benchmark 256^3 D3Q19: reference %.0f MLUPS, case mode %.0f MLUPS; u rms %.2e, du rms %.2e "
          "(rel L2 %.2e), max |drho| %.2e" % (ml_ref, ml_ours, u_rms, du_rms, e, drho))
    assert du_rms < 1e-4 * 0.005 and drho < 1e-5


def test_taylor_green_d3q27_case_matches_reference_program(tmp_path):
    ml_ref = run(os.path.join(REF, "refsim_tgv256_q27"), tmp_path / "ref")
    ml_ours = run(os.path.join(REF, "cases", "tgv256_q27"), tmp_path / "ours")

    def ke(d):
        rows = [l.strip().split(",") for l in open(os.path.join(d, "TEST", "000", "000_totalKineticEnergy.txt"))]
        return {int(r[1]): float(r[2]) for r in rows if len(r) == 3}

    kr, ko = ke(tmp_path / "ref"), ke(tmp_path / "ours")
    assert sorted(kr) == sorted(ko) and len(kr) == 9
    worst = max(abs(ko[s] - kr[s]) / kr[s] for s in kr)
    print("TGV 256^3 D3Q27: reference %.0f MLUPS, case mode %.0f MLUPS; KE worst rel diff %.2e" % (ml_ref, ml_ours, worst))
    assert worst < 2e-5


def write_voxels(path, n):
    """A sphere of radius 9 at the centre and a small blob across the corner of
    the periodic box (its neighbours wrap), as "x,y,z" lines."""
    c = (n - 1) / 2.0
    pts = []
    for z in range(n):
        for y in range(n):
            for x in range(n):
                if (x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 <= 81.0:
                    pts.append((x, y, z))
    pts += [(0, 0, 0), (n - 1, 0, 0), (0, n - 1, 1), (1, 1, n - 1)]
    with open(path, "w") as f:
        f.write("".join("%d,%d,%d\n" % p for p in pts))


def test_voxel_case_matches_reference_program(tmp_path):
    n = 64
    for who in ("ref", "ours"):
        os.makedirs(tmp_path / who, exist_ok=True)
        write_voxels(tmp_path / who / "sphere.csv", n)
    ml_ref = run(os.path.join(REF, "refsim_voxel64"), tmp_path / "ref")
    ml_ours = run(os.path.join(REF, "cases", "voxel64"), tmp_path / "ours")
    a, b = fields(tmp_path / "ours", n, 500), fields(tmp_path / "ref", n, 500)
    e = u_err(a, b)
    drho = float(np.max(np.abs(a["rho"] - b["rho"])))
    print("voxel 64^3: reference %.0f MLUPS, case mode %.0f MLUPS; u rel L2 %.2e, max |drho| %.2e"
          % (ml_ref or 0, ml_ours or 0, e, drho))
    assert e < 1e-4 and drho < 1e-5


def test_lid_case_bc_snippet_equals_generic_solver(tmp_path):
    run(os.path.join(REF, "cases", "lid64"), tmp_path / "case")
    n = 64
    d = mrlbm.lid_cavity_desc(n, re=100.0, lid_u=0.05)
    dom = mrlbm.Domain(d)
    dom.set_node_types(mrlbm.lid_cavity_node_types(n, n, n, 1))
    dom.init_uniform()
    dom.step(2000)
    dom.save_macr_bin(str(tmp_path / "lib"), "000", 2000)
    base = os.path.join(tmp_path, "lib", "000", "000_")
    lib = {v: np.fromfile(base + "%s002000.bin" % v, dtype=np.float32).reshape(n, n, n) for v in ("rho", "ux", "uy", "uz")}
    case = fields(tmp_path / "case", n, 2000)
    e = u_err(case, lib)
    print("lid64: case's own bc_definition vs generic solver, u rel L2 %.2e" % e)
    assert e < 1e-4


def test_thermal_case_matches_reference_program(tmp_path):
    """rayleighBenard_Periodic (D3Q19 + D3G19, 64 x 64 x 8, 1000 steps)
    compiled unchanged in case mode -- its bc_definition.inc and its
    g_bc_definition.inc, whose walls read fMom[idxMom(threadIdx.x - 1, ...)],
    run inside the step kernel -- against the reference's own program on the
    same case: C and rho agree to FP32 operation order, velocity (a rest state
    up to round-off, |u| ~ 1e-6) in absolute terms against the free-fall
    velocity of the case."""
    run(os.path.join(REF, "refsim_rb64"), tmp_path / "ref")
    run(os.path.join(REF, "cases", "rb64"), tmp_path / "ours")
    shape = (8, 64, 64)
    out = {}
    for who in ("ref", "ours"):
        base = os.path.join(tmp_path / who, "TEST", "000", "000_")
        out[who] = {v: np.fromfile(base + "%s%06d.bin" % (v, 1000), dtype=np.float32).reshape(shape).astype(np.float64)
                    for v in ("rho", "ux", "uy", "uz", "C")}
    a, b = out["ours"], out["ref"]
    c_err = float(np.sqrt(np.sum((a["C"] - b["C"]) ** 2) / np.sum((b["C"] - 1.0) ** 2)))
    const = np.load(os.path.join(ROOT, "tests", "golden", "ref_kat.npz"))["rbp_const"]
    u_scale = 3.0 * np.sqrt(const[2] * (const[5] - const[6]) * 64)
    u_err = max(float(np.max(np.abs(a[k] - b[k]))) for k in ("ux", "uy", "uz")) / u_scale
    rho_err = float(np.max(np.abs(a["rho"] - b["rho"])))
    print("RB case mode vs reference program: C rel L2 %.3e, max|du| / U %.3e, max|drho| %.3e" % (c_err, u_err, rho_err))
    assert c_err < 1e-4 and u_err < 2e-4 and rho_err < 1e-5


def test_bingham_case_matches_reference_program(tmp_path):
    """parallelPlates_D3Q19_turbulent_Bingham (walls in y, periodic x and z,
    Bingham fluid with yield stress Bn U_MAX^2, cuRAND-perturbed log-law
    start; its body force set to 0 in both builds, since the reference's
    kernel drops it) at 32 x 32 x 64 and Re 10, 1000 steps,
    compiled unchanged in case mode against the reference's own program: the
    final fields, and the turbulence statistics its treat_data.inc writes
    at the step-500 report (mean velocity and velocity fluctuations per
    distance from the walls, through the reference's host idxMom layout and
    saveTreatData)."""
    ml_ref = run(os.path.join(REF, "refsim_bingham32"), tmp_path / "ref")
    ml_ours = run(os.path.join(REF, "cases", "bingham32"), tmp_path / "ours")
    shape = (64, 32, 32)
    out = {}
    for who in ("ref", "ours"):
        base = os.path.join(tmp_path / who, "TEST", "001", "001_")
        out[who] = {v: np.fromfile(base + "%s001000.bin" % v, dtype=np.float32).reshape(shape)
                    for v in ("rho", "ux", "uy", "uz")}
    e = u_err(out["ours"], out["ref"])
    drho = float(np.max(np.abs(out["ours"]["rho"] - out["ref"]["rho"])))
    stats = {}
    for name in ("ux_mean", "uy_mean", "uz_mean", "ux_fluct", "uy_fluct", "uz_fluct", "uxuy_fluct", "uxuz_fluct",
                 "uyuz_fluct"):
        rows = []
        for who in ("ref", "ours"):
            with open(os.path.join(tmp_path / who, "TEST", "001", "001_turbulent_%s.txt" % name)) as f:
                lines = [ln.strip() for ln in f if ln.strip()]
            assert len(lines) == 1 and lines[0].startswith("step,500,"), (who, name, lines[:2])
            rows.append(np.array([float(v) for v in lines[0].split(",")[2:]]))
        assert rows[0].shape == rows[1].shape == (16,)
        stats[name] = float(np.max(np.abs(rows[1] - rows[0])) / max(np.max(np.abs(rows[0])), 1e-30))
    print("bingham 32x32x64: reference %.0f MLUPS, case mode %.0f MLUPS; u rel L2 %.2e, max |drho| %.2e; "
          "statistics max rel diff %s" % (ml_ref or 0, ml_ours or 0, e, drho,
                                          ", ".join("%s %.1e" % kv for kv in stats.items())))
    assert e < 1e-4 and drho < 1e-5
    assert max(stats.values()) < 1e-3
