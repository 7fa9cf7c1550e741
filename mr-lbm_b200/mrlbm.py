"""ctypes binding of libmrlbm.so (the C ABI declared in include/mrlbm.h).

This is the host-side mirror of the reference's case interface for Python
callers (tests, bench, scripts).  It loads the in-tree CUDA library and fails
loudly when it is missing; there is no CPU fallback.

Arrays are numpy, x fastest: scalar fields have shape (nz, ny, nx); moment
arrays have shape (nm, nz, ny, nx).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# MRLBM_LIBRARY may name another build of the library (the bounds-check
# build libmrlbm_check.so); default: the in-tree libmrlbm.so
LIB_PATH = os.environ.get("MRLBM_LIBRARY") or os.path.join(HERE, "libmrlbm.so")

D3Q19, D3Q27 = 19, 27
F32, F16, BF16, F16U = 0, 1, 2, 3  # F16U: fp16 with split (two-word) velocity
NEWTONIAN, POWERLAW, BINGHAM = 0, 1, 2

NODE_BULK = 0x00
NODE_SOLID = 0xFF
BC_VELOCITY_WALL = 1 << 8
BC_OUTFLOW = 2 << 8


def BC_VELOCITY_INDEX(k):
    return (int(k) & 3) << 11


# thermal rule of a boundary node (include/mrlbm.h MRLBM_THERMAL_*)
THERMAL_KEEP, THERMAL_DIRICHLET, THERMAL_DIRICHLET_FLUX, THERMAL_ADIABATIC = 0, 1, 2, 3


def THERMAL_RULE(r):
    return (int(r) & 3) << 13


def THERMAL_INDEX(k):
    return (int(k) & 3) << 15


# octant masks of the reference's nodeTypeMap (src/nodeTypeMap.h:10-44)
WEST, EAST, SOUTH, NORTH, BACK, FRONT = 0x55, 0xAA, 0x33, 0xCC, 0x0F, 0xF0

STATUS = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "EIO", 5: "EDIVERGED", 6: "ETIMEDOUT",
          7: "ENOTFOUND", 8: "EBUSY", 9: "ECANCELED", 10: "EBOUNDS"}


class MrlbmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class Desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lattice", C.c_int), ("storage", C.c_int),
        ("periodic", C.c_int * 3),
        ("tau", C.c_double), ("rho0", C.c_double),
        ("force", C.c_double * 3),
        ("bc_velocity", (C.c_double * 3) * 4),
        ("rheology", C.c_int),
        ("nnf_n", C.c_double), ("nnf_k", C.c_double),
        ("nnf_yield", C.c_double), ("nnf_omega_p", C.c_double),
        ("bc_matrix_q", C.c_int),
        ("thermal", C.c_int),
        ("t_diffusivity", C.c_double),
        ("t_reference", C.c_double),
        ("t_gravity_beta", C.c_double * 3),
        ("t_source", C.c_double),
        ("t_wall", C.c_double * 4),
        ("reserved", C.c_int * 8),
    ]


class Sums(C.Structure):
    _fields_ = [("mass", C.c_double), ("momentum", C.c_double * 3), ("kinetic_energy", C.c_double),
                ("fluid_nodes", C.c_double), ("max_speed", C.c_double), ("nonfinite", C.c_double)]

    def as_dict(self):
        return {"mass": self.mass, "momentum": tuple(self.momentum), "kinetic_energy": self.kinetic_energy,
                "fluid_nodes": self.fluid_nodes, "max_speed": self.max_speed, "nonfinite": self.nonfinite}


REQ_LID_CAVITY, REQ_DUCT = 0, 1


# z-slab plane selectors (include/mrlbm.h MRLBM_ZPLANE_* / MRLBM_ZGHOST_*)
ZPLANE_FIRST, ZPLANE_LAST, ZGHOST_BELOW, ZGHOST_ABOVE = 0, 1, 2, 3


class ZPlane(C.Structure):
    _fields_ = [("base", C.c_void_p), ("pair_stride", C.c_longlong), ("bytes", C.c_longlong),
                ("npairs", C.c_int), ("device", C.c_int)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int), ("n", C.c_int), ("re", C.c_double), ("lid_u", C.c_double),
                ("nnf_n", C.c_double), ("tau", C.c_double), ("force_z", C.c_double),
                ("solid_fraction", C.c_double), ("seed", C.c_uint64), ("arrival", C.c_double)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("steps", C.c_int), ("residual", C.c_double), ("arrival", C.c_double),
                ("admitted", C.c_double), ("finished", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int), ("active", C.c_int), ("done", C.c_int), ("failed", C.c_int),
                ("hbm_in_use", C.c_double), ("p50_latency", C.c_double), ("p99_latency", C.c_double),
                ("mean_latency", C.c_double), ("solves_per_s", C.c_double), ("lattice_updates", C.c_double)]


_lib = None
FP = C.POINTER(C.c_float)
VP = C.c_void_p


def lib():
    """Load libmrlbm.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libmrlbm.so not built: run python mr-lbm_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.mrlbm_last_error.restype = C.c_char_p
        L.mrlbm_version.restype = C.c_char_p
        sigs = {
            "mrlbm_set_device": [C.c_int],
            "mrlbm_device_count": [C.POINTER(C.c_int)],
            "mrlbm_host_alloc": [C.c_size_t, C.POINTER(VP)],
            "mrlbm_host_free": [VP],
            "mrlbm_domain_create": [C.POINTER(Desc), C.POINTER(VP)],
            "mrlbm_domain_destroy": [VP],
            "mrlbm_domain_bytes": [C.POINTER(Desc), C.POINTER(C.c_size_t)],
            "mrlbm_set_node_types": [VP, C.POINTER(C.c_uint32)],
            "mrlbm_init_flow": [VP, FP, FP, FP, FP],
            "mrlbm_init_uniform": [VP, C.POINTER(C.c_double)],
            "mrlbm_init_taylor_green": [VP, C.c_double, C.c_double],
            "mrlbm_step": [VP, C.c_int],
            "mrlbm_step_graph": [VP, C.c_int],
            "mrlbm_time_steps": [VP, C.c_int, FP],
            "mrlbm_synchronize": [VP],
            "mrlbm_get_step": [VP, C.POINTER(C.c_int)],
            "mrlbm_num_moments": [VP, C.POINTER(C.c_int)],
            "mrlbm_get_moments_ref_layout": [VP, FP],
            "mrlbm_set_moments_ref_layout": [VP, FP],
            "mrlbm_get_moments": [VP, FP],
            "mrlbm_set_moments": [VP, FP],
            "mrlbm_get_macr": [VP, FP, FP, FP, FP, FP],
            "mrlbm_reduce_fp64": [VP, C.POINTER(Sums)],
            "mrlbm_residual": [VP, C.POINTER(C.c_double)],
            "mrlbm_save_checkpoint": [VP, C.c_char_p, C.c_char_p, C.c_int],
            "mrlbm_load_checkpoint": [VP, C.c_char_p, C.c_char_p, C.POINTER(C.c_int)],
            "mrlbm_save_macr_bin": [VP, C.c_char_p, C.c_char_p, C.c_int],
            "mrlbm_save_vtk": [VP, C.c_char_p, C.c_char_p, C.c_int],
            "mrlbm_save_info": [VP, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_double],
            "mrlbm_info_text": [C.POINTER(Desc), C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_char_p, C.c_size_t,
                                C.POINTER(C.c_size_t)],
            "mrlbm_voxel_mark_csv": [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_longlong)],
            "mrlbm_voxel_resolve": [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32)],
            "mrlbm_voxel_node_types": [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_int),
                                       C.POINTER(C.c_uint32)],
            "mrlbm_lid_cavity_node_types": [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32)],
            "mrlbm_bc_class_info": [C.c_int, C.c_int, C.c_uint32, C.POINTER((C.c_double * 3) * 4), C.c_double,
                                    FP, C.POINTER(C.c_uint32)],
            "mrlbm_batch_create": [C.c_int, C.c_int, C.POINTER(VP)],
            "mrlbm_batch_destroy": [VP],
            "mrlbm_batch_add": [VP, C.POINTER(Desc), C.POINTER(C.c_int)],
            "mrlbm_batch_remove": [VP, C.c_int],
            "mrlbm_batch_domain": [VP, C.c_int, C.POINTER(VP)],
            "mrlbm_batch_step": [VP, C.c_int],
            "mrlbm_batch_synchronize": [VP],
            "mrlbm_batch_time_steps": [VP, C.c_int, FP],
            "mrlbm_batch_info": [VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)],
            "mrlbm_batch_autotune": [VP],
            "mrlbm_batch_set_rows": [VP, C.c_int],
            "mrlbm_batch_get_rows": [VP, C.POINTER(C.c_int)],
            "mrlbm_batch_chunk_for": [VP, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)],
            "mrlbm_server_create": [C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(VP)],
            "mrlbm_server_destroy": [VP],
            "mrlbm_server_submit": [VP, C.POINTER(Request), C.POINTER(C.c_int)],
            "mrlbm_server_cancel": [VP, C.c_int],
            "mrlbm_server_tick": [VP, C.POINTER(C.c_int)],
            "mrlbm_server_result": [VP, C.c_int, C.POINTER(RequestResult)],
            "mrlbm_server_moments": [VP, C.c_int, FP, C.c_size_t],
            "mrlbm_server_release": [VP, C.c_int],
            "mrlbm_server_stats_get": [VP, C.POINTER(ServerStats)],
            "mrlbm_server_now": [VP, C.POINTER(C.c_double)],
            "mrlbm_server_inject_nan": [VP, C.c_int],
            "mrlbm_server_keep_results": [VP, C.c_int],
            "mrlbm_server_set_capacity": [VP, C.c_double],
            "mrlbm_request_domain": [C.POINTER(Request), C.c_int, C.POINTER(VP)],
            "mrlbm_request_describe": [C.POINTER(Request), C.c_int, C.POINTER(Desc), C.POINTER(C.c_uint32)],
            "mrlbm_reduce_fp64_ref_layout_noalloc": [VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, VP,
                                                     C.POINTER(Sums)],
            "mrlbm_selftest_bounded_wait": [C.c_uint, C.POINTER(C.c_double)],
            "mrlbm_set_stream": [VP, VP],
            "mrlbm_set_z_chunk": [VP, C.c_int],
            "mrlbm_set_tile_order": [VP, C.c_int],
            "mrlbm_nccl_unique_id": [VP],
            "mrlbm_nccl_comm_init": [C.c_int, VP, C.c_int, C.POINTER(VP)],
            "mrlbm_nccl_comm_destroy": [VP],
            "mrlbm_zslab_exchange_nccl": [VP, VP, C.c_int, C.c_int],
            "mrlbm_get_z_chunk": [VP, C.POINTER(C.c_int)],
            "mrlbm_get_stream": [VP, C.POINTER(VP)],
            "mrlbm_zslab_plane": [VP, C.c_int, C.POINTER(ZPlane)],
            "mrlbm_zslab_copy": [VP, C.c_int, VP, C.c_int],
        }
        for name, args in sigs.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise MrlbmError(status, lib().mrlbm_last_error().decode())


def _fp(a):
    return a.ctypes.data_as(FP)


def selftest_bounded_wait(polls):
    """Run the bounded-wait self-test; returns (status, seconds)."""
    sec = C.c_double()
    st = lib().mrlbm_selftest_bounded_wait(C.c_uint(int(polls)), C.byref(sec))
    return st, sec.value


def set_device(dev):
    check(lib().mrlbm_set_device(int(dev)))


def device_count():
    n = C.c_int()
    check(lib().mrlbm_device_count(C.byref(n)))
    return n.value


class PinnedArray:
    """numpy view over page-locked host memory from mrlbm_host_alloc."""

    def __init__(self, shape, dtype=np.float32):
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = VP()
        check(lib().mrlbm_host_alloc(self.nbytes, C.byref(self.ptr)))
        buf = (C.c_char * self.nbytes).from_address(self.ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            lib().mrlbm_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        self.free()


def make_desc(nx, ny, nz, lattice=D3Q19, storage=F32, periodic=(1, 1, 1), tau=0.8, rho0=1.0,
              force=(0.0, 0.0, 0.0), bc_velocity=None, rheology=NEWTONIAN, nnf_n=1.0, nnf_k=0.0,
              nnf_yield=0.0, nnf_omega_p=0.0, bc_matrix_q=0, thermal=None):
    """thermal: None, or a dict with diffusivity, reference (1.0), gravity_beta
    (3 values), source (0) and wall (up to 4 values): the thermal scalar."""
    d = Desc()
    d.nx, d.ny, d.nz = nx, ny, nz
    d.lattice, d.storage = lattice, storage
    for a in range(3):
        d.periodic[a] = int(periodic[a])
        d.force[a] = float(force[a])
    d.tau, d.rho0 = float(tau), float(rho0)
    if bc_velocity is not None:
        for k, v in enumerate(bc_velocity):
            for a in range(3):
                d.bc_velocity[k][a] = float(v[a])
    d.rheology = rheology
    d.nnf_n, d.nnf_k, d.nnf_yield, d.nnf_omega_p = nnf_n, nnf_k, nnf_yield, nnf_omega_p
    d.bc_matrix_q = bc_matrix_q
    if thermal is not None:
        d.thermal = 1
        d.t_diffusivity = float(thermal["diffusivity"])
        d.t_reference = float(thermal.get("reference", 1.0))
        for a, v in enumerate(thermal.get("gravity_beta", (0.0, 0.0, 0.0))):
            d.t_gravity_beta[a] = float(v)
        d.t_source = float(thermal.get("source", 0.0))
        for k, v in enumerate(thermal.get("wall", ())):
            d.t_wall[k] = float(v)
    return d


def domain_bytes(desc):
    n = C.c_size_t()
    check(lib().mrlbm_domain_bytes(C.byref(desc), C.byref(n)))
    return n.value


class Domain:
    """One MR-LBM domain resident on the current GPU."""

    def __init__(self, desc):
        self.L = lib()
        self.desc = desc
        h = VP()
        check(self.L.mrlbm_domain_create(C.byref(desc), C.byref(h)))
        self.h = h
        nm = C.c_int()
        check(self.L.mrlbm_num_moments(self.h, C.byref(nm)))
        self.nm = nm.value
        self.shape = (desc.nz, desc.ny, desc.nx)

    def close(self):
        if getattr(self, "h", None):
            self.L.mrlbm_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- setup
    def set_node_types(self, nt):
        nt = np.ascontiguousarray(nt, dtype=np.uint32)
        assert nt.size == np.prod(self.shape)
        check(self.L.mrlbm_set_node_types(self.h, nt.ctypes.data_as(C.POINTER(C.c_uint32))))

    def init_flow(self, rho, ux, uy, uz):
        a = [np.ascontiguousarray(v, dtype=np.float32).reshape(-1) for v in (rho, ux, uy, uz)]
        check(self.L.mrlbm_init_flow(self.h, *[_fp(v) for v in a]))

    def init_uniform(self, u0=(0.0, 0.0, 0.0)):
        u = (C.c_double * 3)(*u0)
        check(self.L.mrlbm_init_uniform(self.h, u))

    def init_taylor_green(self, u0, L):
        check(self.L.mrlbm_init_taylor_green(self.h, float(u0), float(L)))

    # -- stepping
    def step(self, n=1):
        check(self.L.mrlbm_step(self.h, int(n)))

    def step_graph(self, n):
        check(self.L.mrlbm_step_graph(self.h, int(n)))

    def time_steps(self, n):
        ms = C.c_float()
        check(self.L.mrlbm_time_steps(self.h, int(n), C.byref(ms)))
        return ms.value

    def set_z_chunk(self, lz):
        """z planes per CTA of the step (0: automatic); results do not depend on it."""
        check(self.L.mrlbm_set_z_chunk(self.h, int(lz)))

    def set_tile_order(self, on):
        """Tile-ordered steps (True, the default): a step may start while the
        one before it finishes, each tile waiting for its neighbours only;
        False orders whole launches.  Results do not depend on it."""
        check(self.L.mrlbm_set_tile_order(self.h, 1 if on else 0))

    def z_chunk(self):
        v = C.c_int()
        check(self.L.mrlbm_get_z_chunk(self.h, C.byref(v)))
        return v.value

    def synchronize(self):
        check(self.L.mrlbm_synchronize(self.h))

    def set_stream(self, stream):
        """Queue the domain's work on `stream` (an integer cudaStream_t of the
        domain's device, e.g. torch.cuda.current_stream().cuda_stream); None
        or 0 returns to the domain's own stream."""
        check(self.L.mrlbm_set_stream(self.h, C.c_void_p(stream or None)))

    def get_stream(self):
        s = VP()
        check(self.L.mrlbm_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def zplane(self, which):
        """Device address, pair stride, bytes per pair and pair count of a z
        plane of the buffer the next step reads (ZPLANE_* / ZGHOST_*)."""
        z = ZPlane()
        check(self.L.mrlbm_zslab_plane(self.h, int(which), C.byref(z)))
        return {"base": z.base or 0, "pair_stride": z.pair_stride, "bytes": z.bytes, "npairs": z.npairs,
                "device": z.device}

    @property
    def step_count(self):
        s = C.c_int()
        check(self.L.mrlbm_get_step(self.h, C.byref(s)))
        return s.value

    # -- data
    def moments(self):
        m = np.empty((self.nm,) + self.shape, dtype=np.float32)
        check(self.L.mrlbm_get_moments(self.h, _fp(m)))
        return m

    def set_moments(self, m):
        m = np.ascontiguousarray(m, dtype=np.float32)
        check(self.L.mrlbm_set_moments(self.h, _fp(m)))

    def moments_ref_layout(self):
        m = np.empty(self.nm * int(np.prod(self.shape)), dtype=np.float32)
        check(self.L.mrlbm_get_moments_ref_layout(self.h, _fp(m)))
        return m

    def set_moments_ref_layout(self, m):
        m = np.ascontiguousarray(m, dtype=np.float32)
        check(self.L.mrlbm_set_moments_ref_layout(self.h, _fp(m)))

    def macr(self):
        out = [np.empty(self.shape, dtype=np.float32) for _ in range(4)]
        check(self.L.mrlbm_get_macr(self.h, *[_fp(v) for v in out], None))
        return out

    def sums(self):
        s = Sums()
        check(self.L.mrlbm_reduce_fp64(self.h, C.byref(s)))
        return s.as_dict()

    def residual(self):
        r = C.c_double()
        check(self.L.mrlbm_residual(self.h, C.byref(r)))
        return r.value

    # -- files
    def save_checkpoint(self, path, sim_id, step):
        check(self.L.mrlbm_save_checkpoint(self.h, path.encode(), sim_id.encode(), int(step)))

    def load_checkpoint(self, path, sim_id):
        s = C.c_int()
        check(self.L.mrlbm_load_checkpoint(self.h, path.encode(), sim_id.encode(), C.byref(s)))
        return s.value

    def save_macr_bin(self, path, sim_id, step):
        check(self.L.mrlbm_save_macr_bin(self.h, path.encode(), sim_id.encode(), int(step)))

    def save_vtk(self, path, sim_id, step):
        check(self.L.mrlbm_save_vtk(self.h, path.encode(), sim_id.encode(), int(step)))

    def save_info(self, path, sim_id, case_name, nsteps, mlups):
        check(self.L.mrlbm_save_info(self.h, path.encode(), sim_id.encode(), case_name.encode(), int(nsteps),
                                     float(mlups)))


class _Member(Domain):
    """A domain owned by a batch: set up and read back like a Domain, stepped by the batch."""

    def __init__(self, batch, mid, handle, desc):
        self.L = lib()
        self.desc = desc
        self.h = handle
        self.batch = batch
        self.id = mid
        nm = C.c_int()
        check(self.L.mrlbm_num_moments(self.h, C.byref(nm)))
        self.nm = nm.value
        self.shape = (desc.nz, desc.ny, desc.nx)

    def close(self):
        self.h = None  # owned by the batch

    def step(self, n=1):
        raise MrlbmError(1, "batch members are stepped by their batch")

    def __getattribute__(self, name):
        # every single-domain call first waits for the batch's queued steps
        if name in ("moments", "set_moments", "moments_ref_layout", "set_moments_ref_layout", "macr", "sums",
                    "residual", "save_checkpoint", "load_checkpoint", "save_macr_bin", "save_info",
                    "set_node_types", "init_flow", "init_uniform", "init_taylor_green"):
            object.__getattribute__(self, "batch").synchronize()
        return object.__getattribute__(self, name)


class Batch:
    """Many domains advanced together by the persistent batched kernel."""

    def __init__(self, lattice=D3Q19, storage=F32):
        self.L = lib()
        h = VP()
        check(self.L.mrlbm_batch_create(lattice, storage, C.byref(h)))
        self.h = h
        self.members = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.mrlbm_batch_destroy(self.h)
            self.h = None
            self.members = {}

    def __del__(self):
        self.close()

    def add(self, desc):
        i = C.c_int()
        check(self.L.mrlbm_batch_add(self.h, C.byref(desc), C.byref(i)))
        d = VP()
        check(self.L.mrlbm_batch_domain(self.h, i.value, C.byref(d)))
        m = _Member(self, i.value, d, desc)
        self.members[i.value] = m
        return m

    def remove(self, member):
        check(self.L.mrlbm_batch_remove(self.h, member.id))
        self.members.pop(member.id, None)
        member.h = None

    def member(self, mid):
        d = VP()
        check(self.L.mrlbm_batch_domain(self.h, mid, C.byref(d)))
        return self.members[mid]

    def step(self, n=1):
        check(self.L.mrlbm_batch_step(self.h, int(n)))

    def synchronize(self):
        check(self.L.mrlbm_batch_synchronize(self.h))

    def time_steps(self, n):
        ms = C.c_float()
        check(self.L.mrlbm_batch_time_steps(self.h, int(n), C.byref(ms)))
        return ms.value

    def info(self):
        m, i, n = C.c_int(), C.c_int(), C.c_longlong()
        check(self.L.mrlbm_batch_info(self.h, C.byref(m), C.byref(i), C.byref(n)))
        return {"members": m.value, "items": i.value, "nodes": n.value}

    def autotune(self):
        check(self.L.mrlbm_batch_autotune(self.h))

    def set_rows(self, rows):
        """Tile height of the batch kernel: 8 or 14 interior rows per CTA."""
        check(self.L.mrlbm_batch_set_rows(self.h, int(rows)))

    def rows(self):
        v = C.c_int()
        check(self.L.mrlbm_batch_get_rows(self.h, C.byref(v)))
        return v.value

    def chunk_for(self, nx, ny, nz):
        lz = C.c_int()
        check(self.L.mrlbm_batch_chunk_for(self.h, nx, ny, nz, C.byref(lz)))
        return lz.value


def make_request(kind, n, re=100.0, lid_u=0.0, nnf_n=1.0, tau=0.0, force_z=0.0, solid_fraction=0.05, seed=0,
                 arrival=-1.0):
    r = Request()
    r.kind, r.n, r.re, r.lid_u, r.nnf_n, r.tau = kind, n, re, lid_u, nnf_n, tau
    r.force_z, r.solid_fraction, r.seed, r.arrival = force_z, solid_fraction, seed, arrival
    return r


class _Owned(Domain):
    """A Domain built by the library from a request description."""

    def __init__(self, handle, n, nm):
        self.L = lib()
        self.h = handle
        self.nm = nm
        self.shape = (n, n, n)
        self.desc = None


def request_domain(req, storage=F16):
    """A standalone Domain set up exactly as the server sets up `req`."""
    h = VP()
    check(lib().mrlbm_request_domain(C.byref(req), storage, C.byref(h)))
    nm = C.c_int()
    check(lib().mrlbm_num_moments(h, C.byref(nm)))
    return _Owned(h, req.n, nm.value)


def info_text(desc, sim_id, case_name=None, nsteps=0, mlups=0.0):
    """The reference-format _info.txt text for a description (host only)."""
    n = C.c_size_t()
    cn = case_name.encode() if case_name else None
    check(lib().mrlbm_info_text(C.byref(desc), sim_id.encode(), cn, int(nsteps), float(mlups), None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(lib().mrlbm_info_text(C.byref(desc), sim_id.encode(), cn, int(nsteps), float(mlups), buf, n.value + 1,
                                C.byref(n)))
    return buf.value.decode()


def request_describe(req, storage=F16):
    """(Desc, node types (n, n, n) uint32 z-y-x) that the server builds for `req` (host only)."""
    d = Desc()
    nt = np.zeros((req.n, req.n, req.n), dtype=np.uint32)
    check(lib().mrlbm_request_describe(C.byref(req), storage, C.byref(d), nt.ctypes.data_as(C.POINTER(C.c_uint32))))
    return d, nt


def nccl_unique_id():
    """A 128-byte NCCL unique id (bytes) for mrlbm_nccl_comm_init on every rank."""
    b = C.create_string_buffer(128)
    check(lib().mrlbm_nccl_unique_id(C.cast(b, VP)))
    return b.raw


class NcclComm:
    """A communicator of the library's NCCL (mrlbm_nccl_comm_init) on the current device."""

    def __init__(self, nranks, uid, rank):
        self.h = VP()
        buf = C.create_string_buffer(bytes(uid), 128)
        check(lib().mrlbm_nccl_comm_init(int(nranks), C.cast(buf, VP), int(rank), C.byref(self.h)))

    def close(self):
        if self.h:
            check(lib().mrlbm_nccl_comm_destroy(self.h))
            self.h = VP()


class Server:
    """Continuous-batching solve server (mrlbm_server_* in include/mrlbm.h)."""

    def __init__(self, storage=F16, hbm_budget=150e9, max_active=512, steps_per_tick=100, residual_tol=1e-6,
                 max_steps=20000, keep_results=False, capacity_nodes=0):
        self.L = lib()
        h = VP()
        check(self.L.mrlbm_server_create(storage, float(hbm_budget), int(max_active), int(steps_per_tick),
                                         float(residual_tol), int(max_steps), C.byref(h)))
        self.h = h
        if keep_results:
            check(self.L.mrlbm_server_keep_results(self.h, 1))
        if capacity_nodes:
            check(self.L.mrlbm_server_set_capacity(self.h, float(capacity_nodes)))

    def close(self):
        if getattr(self, "h", None):
            self.L.mrlbm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, req):
        rid = C.c_int()
        check(self.L.mrlbm_server_submit(self.h, C.byref(req), C.byref(rid)))
        return rid.value

    def cancel(self, rid):
        check(self.L.mrlbm_server_cancel(self.h, rid))

    def tick(self):
        a = C.c_int()
        check(self.L.mrlbm_server_tick(self.h, C.byref(a)))
        return a.value

    def result(self, rid):
        r = RequestResult()
        check(self.L.mrlbm_server_result(self.h, rid, C.byref(r)))
        return {"status": r.status, "steps": r.steps, "residual": r.residual, "arrival": r.arrival,
                "admitted": r.admitted, "finished": r.finished}

    def moments(self, rid, n, nm=10):
        m = np.empty((nm, n, n, n), dtype=np.float32)
        check(self.L.mrlbm_server_moments(self.h, rid, _fp(m), m.size))
        return m

    def release(self, rid):
        check(self.L.mrlbm_server_release(self.h, rid))

    def stats(self):
        s = ServerStats()
        check(self.L.mrlbm_server_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def now(self):
        t = C.c_double()
        check(self.L.mrlbm_server_now(self.h, C.byref(t)))
        return t.value

    def inject_nan(self, rid):
        check(self.L.mrlbm_server_inject_nan(self.h, rid))


def bc_class_info(lattice, node_type, bc_velocity, omega0, bc_matrix_q=0):
    """Host-built moment-BC data of one node type (see mrlbm_bc_class_info)."""
    uv = ((C.c_double * 3) * 4)()
    for k, v in enumerate(bc_velocity or []):
        for a in range(3):
            uv[k][a] = float(v[a])
    out = np.zeros(67, dtype=np.float32)
    known = C.c_uint32()
    check(lib().mrlbm_bc_class_info(lattice, bc_matrix_q, int(node_type), C.byref(uv), float(omega0), _fp(out),
                                    C.byref(known)))
    return out, known.value


def reduce_ref_layout_noalloc(fmom_device_ptr, nx, ny, nz, num_moments, rho0=1.0, stream=0):
    """FP64 sums of a caller-owned FP32 device field in the reference's idxMom
    layout, computed without any allocation (a static per-device scratch
    array; calls on one device must not overlap).  fmom_device_ptr and stream
    are raw addresses (int)."""
    s = Sums()
    check(lib().mrlbm_reduce_fp64_ref_layout_noalloc(VP(fmom_device_ptr), int(nx), int(ny), int(nz),
                                                      int(num_moments), float(rho0), VP(stream), C.byref(s)))
    return s.as_dict()


def lid_cavity_node_types(nx, ny, nz, lid_velocity_index=1):
    out = np.empty((nz, ny, nx), dtype=np.uint32)
    check(lib().mrlbm_lid_cavity_node_types(nx, ny, nz, lid_velocity_index,
                                           out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out


def voxel_node_types(solid, periodic):
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = solid.shape
    out = np.empty((nz, ny, nx), dtype=np.uint32)
    per = (C.c_int * 3)(*[int(p) for p in periodic])
    check(lib().mrlbm_voxel_node_types(nx, ny, nz, solid.ctypes.data_as(C.POINTER(C.c_uint8)), per,
                                      out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out


def lid_cavity_desc(n, re=100.0, lid_u=0.05, storage=F32, lattice=D3Q19, ny=None, nz=None):
    """The reference's lid-driven cavity constants (src/cases/lidDrivenCavity_3D/
    constants.inc:35-36): nu = U * NX / Re, tau = 1/2 + 3 nu."""
    nx = n
    ny = ny or n
    nz = nz or n
    visc = lid_u * nx / re
    tau = 0.5 + 3.0 * visc
    return make_desc(nx, ny, nz, lattice=lattice, storage=storage, periodic=(0, 0, 0), tau=tau,
                     bc_velocity=[(0, 0, 0), (lid_u, 0, 0), (0, 0, 0), (0, 0, 0)])
