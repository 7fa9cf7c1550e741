"""Checkpoint files exchanged with the reference's own program.

The reference's lid-driven cavity (64^3, Re 100, lid 0.05, with the lid's
edges typed as edge walls so both solvers treat the same populations as known)
built for sm_100 by oracle/build_ref_cuda.sh:
  * refsim_lid64_ckpt runs 1000 steps and writes its checkpoint file set after
    step 500 (src/checkpoint.cu:129-186, main.cu:219-262): this library loads
    it, runs the remaining 499 steps, and must end where the reference ends;
    its own checkpoint of the loaded state must hold the same ghost-face
    populations (_fGhost.*) as the reference's, and its legacy VTK file of
    that state must equal the reference's byte for byte (saveVarVTK,
    src/saveData.cu:303-406);
  * this library writes a checkpoint after step 500, refsim_lid64_load starts
    from it (loadSimCheckpoint, src/checkpoint.cu:353-369) and must end where
    this library ends.
The reference reads the step number from a file whose name it builds with
Windows separators (src/checkpoint.cu:321) while it reads the arrays through
POSIX paths; the test gives it that name as a plain file next to the others.
Agreement is to FP32 operation order: relative L2 of u below 1e-4.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import lattice_np
import mrlbm
from test_gpu_reference_build import lid_edges_as_walls

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
N = 64
STEP_NAME = "..\\\\bin\\\\TEST\\\\000\\\\checkpoint\\\\_curr_step.bin"   # as src/checkpoint.cu:321 builds it
GHOSTS = ["X_0", "X_1", "Y_0", "Y_1", "Z_0", "Z_1"]


def run_ref(name, workdir):
    exe = os.path.join(REF_DIR, name)
    if not os.path.exists(exe):
        pytest.skip("reference CUDA build missing (oracle/build_ref_cuda.sh needs the reference tree)")
    os.makedirs(os.path.join(workdir, "TEST", "000", "checkpoint"), exist_ok=True)
    r = subprocess.run([exe], cwd=workdir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def fields(base):
    return {v: np.fromfile(base + v + "001000.bin", dtype=np.float32).reshape(N, N, N) for v in ("rho", "ux", "uy", "uz")}


def u_err(a, b):
    return lattice_np.rel_l2(np.stack([a["ux"], a["uy"], a["uz"]]), np.stack([b["ux"], b["uy"], b["uz"]]))


def new_domain():
    dom = mrlbm.Domain(mrlbm.lid_cavity_desc(N, re=100.0, lid_u=0.05))
    dom.set_node_types(lid_edges_as_walls())
    return dom


def test_library_continues_a_reference_checkpoint(tmp_path):
    ref = str(tmp_path / "ref")
    run_ref("refsim_lid64_ckpt", ref)
    ck = os.path.join(ref, "TEST", "000", "checkpoint")
    assert np.fromfile(os.path.join(ck, "_curr_step.bin"), dtype=np.int32)[0] == 500
    dom = new_domain()
    step = dom.load_checkpoint(os.path.join(ref, "TEST"), "000")
    assert step == 501
    # the loaded state written back out: same moments, same ghost faces
    dom.save_checkpoint(str(tmp_path / "lib"), "000", 500)
    mine = os.path.join(tmp_path, "lib", "000", "checkpoint")
    a = np.fromfile(os.path.join(mine, "_fMom.bin"), dtype=np.float32)
    b = np.fromfile(os.path.join(ck, "_fMom.bin"), dtype=np.float32)
    assert np.array_equal(a, b)
    for g in GHOSTS:
        ga = np.fromfile(os.path.join(mine, "_fGhost.%s.bin" % g), dtype=np.float32)
        gb = np.fromfile(os.path.join(ck, "_fGhost.%s.bin" % g), dtype=np.float32)
        assert ga.size == gb.size
        d = float(np.max(np.abs(ga.astype(np.float64) - gb)))
        print("ghost face %s: %d populations, max |diff| %.2e (max |f| %.2e)" % (g, ga.size, d, np.max(np.abs(gb))))
        assert d < 1e-6
    # the legacy VTK of the same state, byte for byte as the reference's saveVarVTK
    dom.save_vtk(str(tmp_path / "lib"), "000", 500)
    with open(os.path.join(tmp_path, "lib", "000", "000_vtk000500.vtk"), "rb") as f:
        mine_vtk = f.read()
    with open(os.path.join(ref, "TEST", "000", "000_vtk000500.vtk"), "rb") as f:
        ref_vtk = f.read()
    assert len(mine_vtk) == len(ref_vtk) and mine_vtk == ref_vtk
    dom.step(1000 - step)
    dom.save_macr_bin(str(tmp_path / "lib"), "000", 1000)
    dom.close()
    e = u_err(fields(os.path.join(tmp_path, "lib", "000", "000_")), fields(os.path.join(ref, "TEST", "000", "000_")))
    print("reference checkpoint at 500 continued here to 1000: u rel L2 vs the reference's own run %.2e" % e)
    assert e < 1e-4


def test_reference_continues_a_library_checkpoint(tmp_path):
    work = str(tmp_path / "ref")
    dom = new_domain()
    dom.init_uniform()
    dom.step(501)               # the reference's loop indices 0..500
    dom.save_checkpoint(os.path.join(work, "TEST"), "000", 500)
    ck = os.path.join(work, "TEST", "000", "checkpoint")
    shutil.copy(os.path.join(ck, "_curr_step.bin"), os.path.join(work, STEP_NAME))
    out = run_ref("refsim_lid64_load", work)
    assert "Loaded checkpoint" in out
    dom.step(499)
    dom.save_macr_bin(str(tmp_path / "lib"), "000", 1000)
    dom.close()
    e = u_err(fields(os.path.join(tmp_path, "lib", "000", "000_")), fields(os.path.join(work, "TEST", "000", "000_")))
    print("library checkpoint at 500 continued by the reference to 1000: u rel L2 vs this library's run %.2e" % e)
    assert e < 1e-4


@pytest.mark.parametrize("storage", [mrlbm.F32, mrlbm.F16U])
def test_plain_flow_checkpoint_round_trip(tmp_path, storage):
    """A periodic Taylor-Green flow saved after 20 steps and loaded into a new
    domain continues exactly as the original (FP32 storage: the checkpoint's
    FP32 moments are the stored values; split-velocity storage: the loaded
    words round back to the same fp16 words)."""
    nx, ny, nz = 48, 40, 32
    d = mrlbm.make_desc(nx, ny, nz, lattice=27, storage=storage, tau=0.56)
    a = mrlbm.Domain(d)
    a.init_taylor_green(0.04, ny / (2 * np.pi))
    a.step(20)
    a.save_checkpoint(str(tmp_path), "007", 19)
    b = mrlbm.Domain(d)
    assert b.load_checkpoint(str(tmp_path), "007") == 20
    np.testing.assert_array_equal(b.moments(), a.moments())
    a.step(10)
    b.step(10)
    np.testing.assert_array_equal(b.moments(), a.moments())
    a.close()
    b.close()
