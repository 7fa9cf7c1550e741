"""ctypes access to the test-only oracle (oracle/liboracle.so) and to the
reference's host-compiled per-node snippets (oracle/_ref/libref_kat.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg import this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
ORACLE_F32_SO = os.path.join(ORACLE_DIR, "liboracle_f32.so")
REF_KAT_SO = os.path.join(ORACLE_DIR, "_ref", "libref_kat.so")

NEWTONIAN, POWERLAW, BINGHAM = 0, 1, 2

D = C.POINTER(C.c_double)


class OrcDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("q", C.c_int),
        ("periodic", C.c_int * 3),
        ("tau", C.c_double), ("rho0", C.c_double),
        ("force", C.c_double * 3),
        ("bc_velocity", (C.c_double * 3) * 4),
        ("rheology", C.c_int),
        ("n_index", C.c_double), ("k_consistency", C.c_double),
        ("yield_stress", C.c_double), ("omega_p", C.c_double),
        ("exterior", C.c_double * 10),
        ("bc_matrix_q", C.c_int),
        ("thermal", C.c_int),
        ("t_alpha", C.c_double),
        ("t_reference", C.c_double),
        ("t_gbeta", C.c_double * 3),
        ("t_source", C.c_double),
        ("t_wall", C.c_double * 4),
    ]


def _ptr(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


_libs = {}


def lib(fp32=False):
    """The FP64 oracle, or with fp32=True the same restatement built with FP32
    arithmetic and storage (the round-off yardstick)."""
    so = ORACLE_F32_SO if fp32 else ORACLE_SO
    if so not in _libs:
        if not os.path.exists(so):
            subprocess.check_call(["make", "-s", os.path.basename(so)], cwd=ORACLE_DIR)
        L = C.CDLL(so)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcDesc)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_num_moments.argtypes = [C.c_void_p]
        L.orc_set_node_types.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
        L.orc_set_moments.argtypes = [C.c_void_p, D]
        L.orc_get_moments.argtypes = [C.c_void_p, D]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_init_from_macro.argtypes = [C.c_void_p, D, D, D, D, C.c_int]
        L.orc_sums.argtypes = [C.c_void_p, D]
        L.orc_threads.restype = C.c_int
        _libs[so] = L
        if fp32:   # its per-node functions take float arguments; only the domain API is used
            return L
        L.orc_reconstruct.argtypes = [C.c_int, C.c_double, D, D]
        L.orc_bulk_moments.argtypes = [C.c_int, D, D]
        L.orc_known_mask.argtypes = [C.c_int, C.c_uint32]
        L.orc_known_mask.restype = C.c_uint32
        L.orc_bc_solve.argtypes = [C.c_int, C.c_int, C.c_uint32, D, C.c_double, D, D]
        L.orc_nnf_powerlaw.argtypes = [C.c_double] * 5
        L.orc_nnf_powerlaw.restype = C.c_double
        L.orc_nnf_bingham.argtypes = [C.c_double] * 3
        L.orc_nnf_bingham.restype = C.c_double
        L.orc_collide.argtypes = [C.POINTER(OrcDesc), D, C.c_double, D, C.c_int]
        L.orc_thermal_coef.argtypes = [C.c_double]
        L.orc_thermal_coef.restype = C.c_double
        L.orc_reconstruct_g.argtypes = [C.c_double, C.c_double, D, D, D]
        L.orc_sums_g.argtypes = [D, C.c_double, D]
        L.orc_face_normal.argtypes = [C.c_uint32, C.POINTER(C.c_int)]
        L.orc_face_normal.restype = C.c_int
    return _libs[so]


def ref_kat():
    """The reference's per-node snippets compiled on the host, or None when
    oracle/_ref was not built (it needs the reference source tree)."""
    if not os.path.exists(REF_KAT_SO):
        return None
    L = C.CDLL(REF_KAT_SO)
    L.ref_reconstruct_q19.argtypes = [D, C.c_double, D]
    L.ref_reconstruct_q27.argtypes = [D, C.c_double, D]
    L.ref_collide.argtypes = [D, C.c_double, D, C.c_double]
    L.ref_bc_lid_q19.argtypes = [C.c_uint, D, C.c_double, C.c_double, D]
    L.ref_bc_voxel_q19.argtypes = [C.c_uint, D, C.c_double, C.c_double, D]
    L.ref_bc_plates_q27.argtypes = [C.c_uint, D, C.c_double, D]
    L.ref_bc_plates_q19.argtypes = [C.c_uint, D, C.c_double, D]
    L.ref_reconstruct_g19.argtypes = [C.c_double, D, D, D]
    L.ref_bc_rb_q19.argtypes = [C.c_uint, D, C.c_double, D]
    L.ref_rb_periodic_constants.argtypes = [D]
    for f in ("ref_bc_lid_q19", "ref_bc_voxel_q19", "ref_bc_plates_q27", "ref_bc_plates_q19"):
        getattr(L, f).restype = C.c_int
    return L


def make_desc(nx, ny, nz, q=19, periodic=(1, 1, 1), tau=0.8, rho0=1.0, force=(0, 0, 0),
              bc_velocity=None, rheology=NEWTONIAN, n_index=1.0, k_consistency=0.0,
              yield_stress=0.0, omega_p=0.0, exterior=None, bc_matrix_q=None, thermal=None):
    """thermal: None, or a dict with alpha, reference, gbeta (3), source, wall (4)."""
    d = OrcDesc()
    d.nx, d.ny, d.nz, d.q = nx, ny, nz, q
    for a in range(3):
        d.periodic[a] = int(periodic[a])
        d.force[a] = float(force[a])
    d.tau, d.rho0 = tau, rho0
    if bc_velocity is not None:
        for k, v in enumerate(bc_velocity):
            for a in range(3):
                d.bc_velocity[k][a] = float(v[a])
    d.rheology = rheology
    d.n_index, d.k_consistency, d.yield_stress, d.omega_p = n_index, k_consistency, yield_stress, omega_p
    if exterior is not None:
        for k in range(10):
            d.exterior[k] = float(exterior[k])
    d.bc_matrix_q = int(bc_matrix_q if bc_matrix_q is not None else (19 if q == 27 else q))
    if thermal is not None:
        d.thermal = 1
        d.t_alpha = float(thermal["alpha"])
        d.t_reference = float(thermal.get("reference", 1.0))
        for a, v in enumerate(thermal.get("gbeta", (0, 0, 0))):
            d.t_gbeta[a] = float(v)
        d.t_source = float(thermal.get("source", 0.0))
        for k, v in enumerate(thermal.get("wall", (1, 1, 1, 1))):
            d.t_wall[k] = float(v)
    return d


class OracleDomain:
    """FP64 oracle domain (fp32=True: the FP32-arithmetic build of the same
    restatement); moments are [nz, ny, nx, nm] (x fastest), float64 at the
    interface in both builds."""

    def __init__(self, desc, fp32=False):
        self.desc = desc
        self.L = lib(fp32)
        self.h = self.L.orc_create(C.byref(desc))
        if not self.h:
            raise MemoryError("oracle allocation failed")
        self.nm = self.L.orc_num_moments(self.h)
        self.shape = (desc.nz, desc.ny, desc.nx)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def set_node_types(self, t):
        t = np.ascontiguousarray(t, dtype=np.uint32).reshape(-1)
        self.L.orc_set_node_types(self.h, _ptr(t, C.c_uint32))

    def set_moments(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        self.L.orc_set_moments(self.h, _ptr(m))

    def moments(self):
        m = np.empty(self.shape + (self.nm,), dtype=np.float64)
        self.L.orc_get_moments(self.h, _ptr(m))
        return m

    def init_from_macro(self, rho, ux, uy, uz, d3q19_sums=True):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, ux, uy, uz)]
        self.L.orc_init_from_macro(self.h, *[_ptr(a) for a in arrs], int(d3q19_sums))

    def step(self, n):
        self.L.orc_step(self.h, int(n))

    def sums(self):
        s = np.zeros(6)
        self.L.orc_sums(self.h, _ptr(s))
        return s
