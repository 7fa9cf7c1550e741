"""Generate tests/golden/ref_kat.npz: known-answer vectors produced by the
reference's own per-node snippets, compiled on the host (oracle/_ref/libref_kat.so,
built by `make -C oracle ref` from the reference source tree).

    python tests/golden/make_golden.py

Contents (all float64):
  recon19_in (N,10) / recon19_out (N,19)   src/colrec/MR_LBM/reconstruction.inc, D3Q19
  recon27_in (N,10) / recon27_out (N,27)   same, D3Q27
  coll_in (N,15) / coll_out (N,10)         src/colrec/MR_LBM/collision.inc
      coll_in = [m0..m9 (scaled, pre-collision), rho, Fx, Fy, Fz, omega]
  lid_type (K,) lid_pops (K,19) lid_omega (K,) lid_umax (K,) lid_out (K,10)
      src/cases/lidDrivenCavity_3D/bc_definition.inc (all 26 wall labels)
  vox_type (254,) vox_pops (254,19) vox_omega (254,) vox_out (254,10)
      src/cases/voxel/bc_definition.inc (all 254 octant masks)
  pl27_type, pl27_pops (.,27), pl27_omega, pl27_out
      src/cases/parallelPlates_D3Q27/bc_definition.inc
  g19_in (N,7) / g19_out (N,19)            src/colrec/G_SCALAR/reconstruction.inc (D3G19)
      g19_in = [C, 3ux, 3uy, 3uz, udx, udy, udz]
  rb_type, rb_pops (.,19), rb_omega, rb_out
      src/cases/rayleighBenard_Periodic/bc_definition.inc (its 6 faces and 12 edges)
  rbp_const (10,)                          src/cases/rayleighBenard_Periodic/constants.inc:
      G_DIFF_FLUC_COEF, T_DIFFUSIVITY, T_gravity_t_beta, VISC, T_REFERENCE, T_HOT,
      T_COLD, gravity_vector[3]
BC outputs are [rho, ux, uy, uz, Pi_xx, Pi_xy, Pi_xz, Pi_yy, Pi_yz, Pi_zz] (unscaled).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import lattice_np  # noqa: E402
import oracle_ffi  # noqa: E402

P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731


def main():
    R = oracle_ffi.ref_kat()
    if R is None:
        raise SystemExit("oracle/_ref/libref_kat.so missing: run `make -C oracle ref` first")
    O = oracle_ffi.lib()
    rng = np.random.default_rng(20261203)
    out = {}

    def pops_near_eq(q, amp=0.05, noise=2e-3):
        m = rng.normal(0.0, amp, 10)
        m[0] = rng.normal(0.0, 0.01)
        f = np.zeros(q)
        O.orc_reconstruct(q, 1.0, P(m), P(f))
        return f + rng.normal(0.0, noise, q) * f

    for q, fn in ((19, R.ref_reconstruct_q19), (27, R.ref_reconstruct_q27)):
        ins = rng.normal(0.0, 0.05, (64, 10))
        outs = np.zeros((64, q))
        for k in range(64):
            fn(P(np.ascontiguousarray(ins[k])), 1.0, P(outs[k]))
        out["recon%d_in" % q], out["recon%d_out" % q] = ins, outs

    cin = np.zeros((64, 15))
    cout = np.zeros((64, 10))
    for k in range(64):
        m = rng.normal(0.0, 0.05, 10)
        rho = 1.0 + rng.normal(0.0, 0.01)
        F = rng.normal(0.0, 1e-4, 3) if k % 2 else np.zeros(3)
        om = rng.uniform(0.5, 1.95)
        cin[k] = np.concatenate([m, [rho], F, [om]])
        mm = m.copy()
        R.ref_collide(P(mm), rho, P(np.ascontiguousarray(F)), om)
        cout[k] = mm
    out["coll_in"], out["coll_out"] = cin, cout

    types, pops, oms, ums, res = [], [], [], [], []
    for name, t in sorted(lattice_np.wall_types().items()):
        for rep in range(3):
            f = pops_near_eq(19)
            om = rng.uniform(0.6, 1.9)
            umax = 0.05
            r = np.zeros(10)
            assert R.ref_bc_lid_q19(t, P(f), om, umax, P(r)) == 1, name
            types.append(t); pops.append(f); oms.append(om); ums.append(umax); res.append(r)
    out["lid_type"] = np.array(types, dtype=np.uint32)
    out["lid_pops"], out["lid_omega"], out["lid_umax"], out["lid_out"] = map(np.array, (pops, oms, ums, res))

    types, pops, oms, res = [], [], [], []
    for t in range(1, 255):
        f = pops_near_eq(19)
        om = rng.uniform(0.6, 1.9)
        r = np.zeros(10)
        assert R.ref_bc_voxel_q19(t, P(f), om, 1.0, P(r)) == 1, t
        types.append(t); pops.append(f); oms.append(om); res.append(r)
    out["vox_type"] = np.array(types, dtype=np.uint32)
    out["vox_pops"], out["vox_omega"], out["vox_out"] = map(np.array, (pops, oms, res))

    types, pops, oms, res = [], [], [], []
    for t in (lattice_np.FACES["SOUTH"], lattice_np.FACES["NORTH"]):
        for rep in range(4):
            f = pops_near_eq(27)
            om = rng.uniform(0.6, 1.9)
            r = np.zeros(10)
            assert R.ref_bc_plates_q27(t, P(f), om, P(r)) == 1
            types.append(t); pops.append(f); oms.append(om); res.append(r)
    out["pl27_type"] = np.array(types, dtype=np.uint32)
    out["pl27_pops"], out["pl27_omega"], out["pl27_out"] = map(np.array, (pops, oms, res))

    gin = np.zeros((64, 7))
    gout = np.zeros((64, 19))
    for k in range(64):
        gin[k, 0] = rng.uniform(0.5, 1.5)
        gin[k, 1:4] = rng.normal(0.0, 0.1, 3)
        gin[k, 4:7] = rng.normal(0.0, 0.05, 3)
        R.ref_reconstruct_g19(gin[k, 0], P(np.ascontiguousarray(gin[k, 1:4])), P(np.ascontiguousarray(gin[k, 4:7])),
                              P(gout[k]))
    out["g19_in"], out["g19_out"] = gin, gout
    rc = np.zeros(10)
    R.ref_rb_periodic_constants(P(rc))
    out["rbp_const"] = rc

    types, pops, oms, res = [], [], [], []
    for name, t in sorted(lattice_np.wall_types().items()):
        if name.count("_") == 2:   # the case lists faces and edges, no corners
            continue
        for rep in range(2):
            f = pops_near_eq(19)
            om = rng.uniform(0.6, 1.9)
            r = np.zeros(10)
            assert R.ref_bc_rb_q19(t, P(f), om, P(r)) == 1, name
            types.append(t); pops.append(f); oms.append(om); res.append(r)
    out["rb_type"] = np.array(types, dtype=np.uint32)
    out["rb_pops"], out["rb_omega"], out["rb_out"] = map(np.array, (pops, oms, res))

    path = os.path.join(HERE, "ref_kat.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
