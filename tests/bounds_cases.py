"""Cases run by the bounds-check test (tests/test_gpu_bounds_check.py) with
both builds of the library: shapes at the edges of the step kernels' column
decomposition (one-node axes; columns one node under, at and over the 32-lane
width and the 8- and 14-row heights; z depths below the chunk) for every
kernel family (bulk, walls, split-velocity fp16, power law with voxel
obstacles, thermal scalar, batched members).

    python tests/bounds_cases.py <out.npz>     # runs with whichever library MRLBM_LIBRARY names
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "mr-lbm_b200"))
import mrlbm  # noqa: E402

STEPS = 6


def _flow(shape, seed):
    rng = np.random.default_rng(seed)
    return (1 + 0.01 * rng.standard_normal(shape), *(0.02 * rng.standard_normal((3,) + shape)))


def _run(d, nt=None, init=None):
    dom = mrlbm.Domain(d)
    if nt is not None:
        dom.set_node_types(nt)
    if init is None:
        dom.init_flow(*_flow((d.nz, d.ny, d.nx), d.nx * 7 + d.ny * 3 + d.nz))
    else:
        init(dom)
    dom.step(STEPS)
    dom.synchronize()     # raises MRLBM_EBOUNDS if the check build skipped an access
    m = dom.moments()
    dom.close()
    return m


def cases():
    out = {}
    for shape, q, st in [((33, 9, 5), 27, mrlbm.F32), ((32, 8, 3), 27, mrlbm.F32), ((1, 12, 10), 19, mrlbm.F32),
                         ((65, 17, 2), 27, mrlbm.F32), ((2, 2, 2), 27, mrlbm.F32), ((31, 7, 4), 19, mrlbm.F16),
                         ((40, 10, 6), 27, mrlbm.F16U)]:
        nx, ny, nz = shape
        out["bulk_%dx%dx%d_q%d_s%d" % (nx, ny, nz, q, st)] = lambda nx=nx, ny=ny, nz=nz, q=q, st=st: _run(
            mrlbm.make_desc(nx, ny, nz, lattice=q, storage=st, tau=0.7))
    for shape, q, st in [((33, 15, 7), 19, mrlbm.F32), ((32, 14, 9), 27, mrlbm.F32), ((29, 13, 6), 19, mrlbm.F16U),
                         ((34, 8, 5), 27, mrlbm.F32), ((31, 17, 3), 19, mrlbm.BF16)]:
        nx, ny, nz = shape

        def cav(nx=nx, ny=ny, nz=nz, q=q, st=st):
            d = mrlbm.lid_cavity_desc(nx, re=100.0, lid_u=0.05, lattice=q, storage=st, ny=ny, nz=nz)
            return _run(d, mrlbm.lid_cavity_node_types(nx, ny, nz, 1), lambda dom: dom.init_uniform())
        out["cavity_%dx%dx%d_q%d_s%d" % (nx, ny, nz, q, st)] = cav

    def duct():
        nx, ny, nz = 20, 18, 12
        rng = np.random.default_rng(4)
        solid = np.zeros((nz, ny, nx), dtype=np.uint8)
        solid[:, 1:-1, 1:-1] = rng.random((nz, ny - 2, nx - 2)) < 0.05
        nt = mrlbm.voxel_node_types(solid, (0, 0, 1))
        d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(0, 0, 1), tau=0.8, force=(0, 0, 2e-5),
                            rheology=mrlbm.POWERLAW, nnf_n=0.7)
        return _run(d, nt, lambda dom: dom.init_uniform())
    out["powerlaw_duct"] = duct

    def thermal():
        nx, ny, nz = 24, 15, 6
        th = dict(diffusivity=0.02, reference=1.0, gravity_beta=(2e-4, 0.0, 0.0), wall=(1.5, 0.5, 1.0, 1.0))
        d = mrlbm.make_desc(nx, ny, nz, lattice=19, periodic=(0, 1, 1), tau=0.56, thermal=th)
        rule = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET)
        nt = np.zeros((nz, ny, nx), dtype=np.uint32)
        nt[:, :, 0] = mrlbm.WEST | rule | mrlbm.THERMAL_INDEX(0)
        nt[:, :, -1] = mrlbm.EAST | rule | mrlbm.THERMAL_INDEX(1)
        return _run(d, nt, lambda dom: dom.init_uniform())
    out["thermal_plates"] = thermal

    def batch():
        b = mrlbm.Batch(mrlbm.D3Q19, mrlbm.F16)
        mem = []
        for nx, ny, nz in ((33, 15, 7), (20, 20, 9)):
            d = mrlbm.lid_cavity_desc(nx, re=100.0, lid_u=0.05, storage=mrlbm.F16, ny=ny, nz=nz)
            m = b.add(d)
            m.set_node_types(mrlbm.lid_cavity_node_types(nx, ny, nz, 1))
            m.init_uniform()
            mem.append(m)
        b.step(STEPS)
        b.synchronize()
        for m in mem:
            m.synchronize()
        res = np.concatenate([m.moments().ravel() for m in mem])
        b.close()
        return res
    out["batch_f16"] = batch
    return out


def run_all():
    return {k: f() for k, f in cases().items()}


if __name__ == "__main__":
    res = run_all()
    np.savez(sys.argv[1], **res)
    print("bounds cases: %d run, library %s" % (len(res), mrlbm.LIB_PATH))
