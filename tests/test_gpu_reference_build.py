"""The library against the reference's own CUDA program (built for sm_100 by
oracle/build_ref_cuda.sh into oracle/_ref), on the same case and inputs.

Lid-driven cavity 64^3, D3Q19, Re 100, lid 0.05, 2000 steps (the reference
binary writes its final macroscopic fields as .bin files, src/saveData.cu):
per-field relative L2 of the library's rho-1 and u against the reference's.
Both sides are FP32; the differences come from operation order only.
"""
import os
import subprocess

import numpy as np
import pytest

import lattice_np
import mrlbm

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFSIM = os.path.join(ROOT, "oracle", "_ref", "refsim_lid64")


def read_bin(path, n):
    a = np.fromfile(path, dtype=np.float32)
    assert a.size == n ** 3, (path, a.size)
    return a.reshape(n, n, n)


@pytest.fixture(scope="module")
def reference_lid64(tmp_path_factory):
    if not os.path.exists(REFSIM):
        pytest.skip("reference CUDA build missing (oracle/build_ref_cuda.sh needs the reference tree)")
    work = tmp_path_factory.mktemp("refsim")
    r = subprocess.run([REFSIM], cwd=work, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    base = os.path.join(work, "TEST", "000", "000_")
    n = 64
    out = {v: read_bin(base + v + "002000.bin", n) for v in ("rho", "ux", "uy", "uz")}
    out["log"] = r.stdout
    return out


def test_lid_cavity_64_matches_reference_build(reference_lid64, tmp_path):
    n = 64
    d = mrlbm.lid_cavity_desc(n, re=100.0, lid_u=0.05)
    dom = mrlbm.Domain(d)
    dom.set_node_types(mrlbm.lid_cavity_node_types(n, n, n, 1))
    dom.init_uniform()
    dom.step(2000)
    dom.save_macr_bin(str(tmp_path), "000", 2000)
    ours = {v: read_bin(os.path.join(tmp_path, "000", "000_" + v + "002000.bin"), n) for v in ("rho", "ux", "uy", "uz")}
    ref = reference_lid64
    e_rho = lattice_np.rel_l2(ours["rho"] - 1.0, ref["rho"] - 1.0)
    u_ours = np.stack([ours["ux"], ours["uy"], ours["uz"]])
    u_ref = np.stack([ref["ux"], ref["uy"], ref["uz"]])
    e_u = lattice_np.rel_l2(u_ours, u_ref)
    e_uinf = lattice_np.rel_linf(u_ours, u_ref)
    print("lid64 vs reference build: rel L2 rho-1 %.3e, u %.3e, u Linf %.3e" % (e_rho, e_u, e_uinf))
    assert e_u < 1e-4 and e_uinf < 1e-3
    assert e_rho < 1e-3
