"""FP64 fixtures of the periodic Taylor-Green vortex on D3Q27 (TEST
INFRASTRUCTURE: runs the FP64 oracle, oracle/liboracle.so, on the host).

    python tests/golden/make_tgv_fixtures.py tgv256       # ~15 min on 8 cores
    python tests/golden/make_tgv_fixtures.py tgv128re400  # ~3 min

tgv256: 256^3, Re 1600, u0 0.04, 1000 steps (src/cases/taylorGreen/
constants.inc, flow_initialization.inc): the FP64 kinetic energy every 100
steps and the stored moments of z planes 0 and 96, every 4th node in x and y
(float32), written to tests/golden/tgv256_fp64.npz.

tgv128re400: 128^3, Re 400 (the same tau as the 512^3 vortex at Re 1600, so
the same viscous damping per step of the rounding noise that 16-bit storage
adds), u0 0.04, 1000 steps: the velocity (3u as stored) of z planes 0, 40 and
80 as float32, written to tests/golden/tgv128re400_fp64.npz.

Both start from the library's initial-state formula (the reference's
flow_initialization.inc, with the D3Q19 second-moment sums of its
gpuInitialization_mom also on D3Q27).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_ffi  # noqa: E402
from tgv_reference import tgv_fields  # noqa: E402


def run(n, re, steps, report):
    u0 = 0.04
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * u0 * L / re
    o = oracle_ffi.OracleDomain(oracle_ffi.make_desc(n, n, n, q=27, tau=tau))
    rho, ux, uy, uz = tgv_fields(n, u0)
    o.init_from_macro(rho, ux, uy, uz)
    ke = [(0, o.sums()[4])]
    t0 = time.time()
    for s in range(report, steps + 1, report):
        o.step(report)
        ke.append((s, o.sums()[4]))
        print("n %d step %d KE %.12e (%.0f s)" % (n, s, ke[-1][1], time.time() - t0), flush=True)
    return o, tau, np.array(ke)


def main(which):
    if which == "tgv256":
        o, tau, ke = run(256, 1600.0, 1000, 100)
        m = o.moments()
        planes = [0, 96]
        sel = np.ascontiguousarray(m[planes][:, ::4, ::4, :]).astype(np.float32)
        np.savez_compressed(os.path.join(HERE, "tgv256_fp64.npz"), n=256, steps=1000, re=1600.0, tau=tau,
                            planes=np.array(planes), stride=4, moments=sel, ke=ke)
    elif which == "tgv128re400":
        o, tau, ke = run(128, 400.0, 1000, 100)
        m = o.moments()
        planes = [0, 40, 80]
        sel = np.ascontiguousarray(m[planes][..., 1:4]).astype(np.float32)
        np.savez_compressed(os.path.join(HERE, "tgv128re400_fp64.npz"), n=128, steps=1000, re=400.0, tau=tau,
                            planes=np.array(planes), u3=sel, ke=ke)
    else:
        raise SystemExit("unknown fixture %s" % which)


if __name__ == "__main__":
    main(sys.argv[1])
