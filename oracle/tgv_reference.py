"""FP64 reference solution of the periodic Taylor-Green vortex (TEST
INFRASTRUCTURE: it runs the oracle, oracle/liboracle.so, on the host).

    python oracle/tgv_reference.py --n 512 --steps 1000 --out tgv512_fp64.npz

D3Q27, N^3 nodes, Re 1600, u0 0.04, L = N / 2pi, tau = 1/2 + 3 u0 L / Re
(src/cases/taylorGreen/constants.inc, flow_initialization.inc), initial field
from the same formula as the library's mrlbm_init_taylor_green.  Writes the
stored moments (oracle layout [z][y][x][10], float32) of a few z planes after
`steps` steps, and the FP64 kinetic energy every `--report` steps: the
reference the storage-precision study (bench.py --workload precision)
compares FP32, FP16 and BF16 storage against.  A 512^3 run holds 21.5 GB of
moments plus a 10.7 GB copy when the planes are read out, and runs at about
15 million lattice updates per second on 8 cores.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tests"))
import oracle_ffi  # noqa: E402


def tgv_fields(n, u0):
    L = n / (2 * np.pi)
    ax = np.arange(n, dtype=np.float64)
    z, y, x = ax[:, None, None], ax[None, :, None], ax[None, None, :]
    rho = 1.0 + (1.0 / (16.0 / 3.0)) * u0 * u0 * (np.cos(2 * x / L) + np.cos(2 * y / L)) * (np.cos(2 * z / L) + 2.0)
    ux = u0 * np.sin(x / L) * np.cos(y / L) * np.cos(z / L)
    uy = -u0 * np.cos(x / L) * np.sin(y / L) * np.cos(z / L)
    shape = (n, n, n)
    return (np.broadcast_to(rho, shape), np.broadcast_to(ux, shape), np.broadcast_to(uy, shape),
            np.zeros(shape))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--report", type=int, default=100)
    ap.add_argument("--planes", default="0,128,256,384")
    ap.add_argument("--re", type=float, default=1600.0)
    ap.add_argument("--u0", type=float, default=0.04)
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    n = args.n
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * args.u0 * L / args.re
    desc = oracle_ffi.make_desc(n, n, n, q=27, tau=tau)
    o = oracle_ffi.OracleDomain(desc)
    rho, ux, uy, uz = tgv_fields(n, args.u0)
    o.init_from_macro(rho, ux, uy, uz)
    del rho, ux, uy, uz
    ke = [(0, o.sums()[4])]
    t0 = time.time()
    for s in range(args.report, args.steps + 1, args.report):
        o.step(args.report)
        ke.append((s, o.sums()[4]))
        print("step %d KE %.10e (%.0f s)" % (s, ke[-1][1], time.time() - t0), flush=True)
    planes = [int(p) for p in args.planes.split(",")]
    m = o.moments()
    sel = np.ascontiguousarray(m[planes]).astype(np.float32)
    del m
    np.savez(args.out, n=n, steps=args.steps, tau=tau, planes=np.array(planes), moments=sel,
             ke=np.array(ke), threads=oracle_ffi.lib().orc_threads(), seconds=time.time() - t0)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
