"""Helpers for GPU-vs-oracle parity runs (test infrastructure)."""
import numpy as np

import lattice_np
import oracle_ffi


def oracle_for(desc, node_types=None, fp32=False):
    """An FP64 oracle domain with the same physics as a library descriptor
    (fp32=True: the FP32-arithmetic build of the oracle)."""
    import mrlbm
    bcv = [tuple(desc.bc_velocity[k][a] for a in range(3)) for k in range(4)]
    kw = dict(q=desc.lattice, periodic=tuple(desc.periodic[a] for a in range(3)), tau=desc.tau, rho0=desc.rho0,
              force=tuple(desc.force[a] for a in range(3)), bc_velocity=bcv, rheology=desc.rheology,
              n_index=desc.nnf_n, k_consistency=desc.nnf_k or desc.rho0 * (desc.tau - 0.5) / 3,
              yield_stress=desc.nnf_yield, omega_p=desc.nnf_omega_p or 1.0 / desc.tau,
              bc_matrix_q=desc.bc_matrix_q or (19 if desc.lattice == 27 else desc.lattice))
    # exterior state: the rest state of the reference's initialisation
    # (D3Q19 second-moment sums also on D3Q27)
    ext = np.zeros(10)
    q = desc.lattice
    w = {19: [1 / 3] + [1 / 18] * 6 + [1 / 36] * 12,
         27: [8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8}[q]
    for k, c in ((4, lattice_np.CX), (7, lattice_np.CY), (9, lattice_np.CZ)):
        ext[k] = 4.5 * (sum(w[i] * c[i] ** 2 for i in range(19)) - 1 / 3)
    kw["exterior"] = ext
    if desc.thermal:
        kw["thermal"] = dict(alpha=desc.t_diffusivity, reference=desc.t_reference,
                             gbeta=tuple(desc.t_gravity_beta[a] for a in range(3)), source=desc.t_source,
                             wall=tuple(desc.t_wall[k] for k in range(4)))
    o = oracle_ffi.OracleDomain(oracle_ffi.make_desc(desc.nx, desc.ny, desc.nz, **kw), fp32=fp32)
    if node_types is not None:
        o.set_node_types(node_types)
    return o


def gpu_to_oracle_layout(m):
    """(nm, nz, ny, nx) float32 -> (nz, ny, nx, nm) float64."""
    return np.moveaxis(np.asarray(m, dtype=np.float64), 0, -1).copy()


# moment groups and the norm each moment's error is measured against:
# rho - rho0 against rho (its FP32 resolution is that of rho itself), each
# velocity component against |u|, each second moment against the group of
# second moments, omega against omega; with the thermal scalar, C against C
# (moment 10) and each flux component against |flux| (moments 11-13).
GROUPS = {0: [0], 1: [1, 2, 3], 2: [1, 2, 3], 3: [1, 2, 3], 4: [4, 5, 6, 7, 8, 9], 5: [4, 5, 6, 7, 8, 9],
          6: [4, 5, 6, 7, 8, 9], 7: [4, 5, 6, 7, 8, 9], 8: [4, 5, 6, 7, 8, 9], 9: [4, 5, 6, 7, 8, 9], 10: [10],
          11: [11, 12, 13], 12: [11, 12, 13], 13: [11, 12, 13]}


def compare(gpu_m, orc_m, fluid=None, rho0=1.0):
    """Per-moment relative L2 / Linf of the GPU moments against the oracle's,
    each normalised by the norm of its moment group (see GROUPS)."""
    g = np.moveaxis(np.asarray(gpu_m, dtype=np.float64), 0, -1)
    o = np.asarray(orc_m, dtype=np.float64)
    if fluid is not None:
        g = g[fluid]
        o = o[fluid]
    res = {}
    for k in range(o.shape[-1]):
        ref = o[..., GROUPS[k]]
        if k == 0:
            ref = ref + rho0
        d = g[..., k] - o[..., k]
        l2 = float(np.sqrt(np.sum(d * d) / max(np.sum(ref * ref) / len(GROUPS[k]), 1e-300)))
        linf = float(np.max(np.abs(d)) / max(np.max(np.abs(ref)), 1e-300))
        res[k] = (l2, linf)
    return res


def velocity_rel_l2(gpu_m, orc_m, fluid=None):
    g = np.moveaxis(np.asarray(gpu_m, dtype=np.float64), 0, -1)[..., 1:4]
    o = np.asarray(orc_m, dtype=np.float64)[..., 1:4]
    if fluid is not None:
        g, o = g[fluid], o[fluid]
    return lattice_np.rel_l2(g, o)
