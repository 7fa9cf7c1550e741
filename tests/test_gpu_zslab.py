"""Z-slab decomposition on one B200: a domain cut into 2-4 slabs (each a
library domain on its own stream, planes moved by mrlbm_zslab_copy) steps to
the same moments, bit for bit, as the undivided domain; the plane views the
NCCL path sends and receives are the domain's boundary planes; one
torch.distributed rank (NCCL, periodic z: the slab is its own neighbour)
matches too.  Multi-rank NCCL runs need several GPUs: their host logic is
covered by tests/test_zslab_host.py with gloo ranks."""
import numpy as np
import pytest

import mrlbm
import zslab

pytestmark = pytest.mark.gpu


def _random_flow(shape, seed, amp=0.03):
    rng = np.random.default_rng(seed)
    rho = (1.0 + 0.01 * rng.standard_normal(shape)).astype(np.float32)
    u = [(amp * rng.standard_normal(shape)).astype(np.float32) for _ in range(3)]
    return rho, u


def _run_both(desc, parts, steps, nt=None, seed=3, init=None):
    shape = (desc.nz, desc.ny, desc.nx)
    rho, u = _random_flow(shape, seed)
    mono = mrlbm.Domain(desc)
    if nt is not None:
        mono.set_node_types(nt)
    if init is None:
        mono.init_flow(rho, *u)
    else:
        init(mono)
    m0 = mono.moments()
    mono.step(steps)
    want = mono.moments()
    mono.close()
    zs = zslab.ZSlabDomain.local(desc, parts)
    if nt is not None:
        zs.set_node_types(nt)
    zs.set_moments(m0)
    zs.step(steps)
    got = zs.moments()
    s = zs.sums()
    zs.close()
    return want, got, s


@pytest.mark.parametrize("parts", [2, 3, 4])
def test_periodic_vortex_d3q27(parts):
    d = mrlbm.make_desc(64, 48, 40, lattice=mrlbm.D3Q27, tau=0.52)
    want, got, s = _run_both(d, parts, 24,
                             init=lambda dom: dom.init_taylor_green(0.04, 40 / (2 * np.pi)))
    assert np.array_equal(got, want)
    assert s["nonfinite"] == 0 and s["fluid_nodes"] == 64 * 48 * 40


def test_lid_cavity_d3q19_walls_on_every_face():
    d = mrlbm.make_desc(40, 36, 33, lattice=mrlbm.D3Q19, periodic=(0, 0, 0), tau=0.6,
                        bc_velocity=[(0.05, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 3)
    nt = mrlbm.lid_cavity_node_types(40, 36, 33, 1)
    want, got, _ = _run_both(d, 3, 30, nt=nt)
    assert np.array_equal(got, want)


def test_half_storage_vortex():
    d = mrlbm.make_desc(48, 40, 36, lattice=mrlbm.D3Q19, storage=mrlbm.F16, tau=0.55)
    want, got, _ = _run_both(d, 2, 20, init=lambda dom: dom.init_taylor_green(0.04, 36 / (2 * np.pi)))
    assert np.array_equal(got, want)


def test_thermal_plates_split_between_them():
    """Rayleigh-Benard layout with the plates normal to z (z = 0 hot, z =
    nz - 1 cold, periodic x and y): the thermal moments 10-13 travel with
    the planes."""
    nx, ny, nz = 32, 24, 20
    th = dict(diffusivity=0.02, reference=1.0, gravity_beta=(0.0, 0.0, 2e-4), wall=(1.5, 0.5, 1.0, 1.0))
    d = mrlbm.make_desc(nx, ny, nz, lattice=mrlbm.D3Q19, periodic=(1, 1, 0), tau=0.56, thermal=th)
    rule = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET)
    nt = np.zeros((nz, ny, nx), dtype=np.uint32)
    nt[0] = mrlbm.BACK | rule | mrlbm.THERMAL_INDEX(0)
    nt[-1] = mrlbm.FRONT | rule | mrlbm.THERMAL_INDEX(1)
    want, got, _ = _run_both(d, 2, 40, nt=nt)
    assert want.shape[0] == 14
    assert np.array_equal(got, want)


def test_plane_views_are_the_boundary_planes():
    """The byte ranges mrlbm_zslab_plane names (what the NCCL path sends and
    receives in place) hold the slab's first / last interior planes and,
    after an exchange, the neighbours' planes."""
    import torch

    d = mrlbm.make_desc(20, 12, 10, lattice=mrlbm.D3Q27, tau=0.6)
    zs = zslab.ZSlabDomain.local(d, 2)
    rho, u = _random_flow((10, 12, 20), 5)
    zs.init_flow(rho, *u)
    zs.synchronize()
    m = zs.moments()                                   # (nm, nz, ny, nx)
    lo, hi = zs.slabs
    XOFF = 4

    def plane(slab, which):
        p = slab.dom.zplane(which)
        assert p["npairs"] == (slab.dom.nm + 1) // 2
        v = [t.view(torch.float32).cpu().numpy() for t in slab.send_buffers(which)]
        pitch = p["bytes"] // 8 // (d.ny + 2)
        out = np.empty((2 * p["npairs"], d.ny, d.nx), dtype=np.float32)
        for k, a in enumerate(v):
            a = a.reshape(d.ny + 2, pitch, 2)[1:-1, XOFF:XOFF + d.nx]
            out[2 * k], out[2 * k + 1] = a[..., 0], a[..., 1]
        return out[:slab.dom.nm]

    assert np.array_equal(plane(lo, mrlbm.ZPLANE_FIRST), m[:, 0])
    assert np.array_equal(plane(lo, mrlbm.ZPLANE_LAST), m[:, lo.z1 - 1])
    assert np.array_equal(plane(hi, mrlbm.ZPLANE_FIRST), m[:, hi.z0])
    # periodic z: slab 0's ghost below is slab 1's last plane, and so on
    assert np.array_equal(plane(lo, mrlbm.ZGHOST_BELOW), m[:, -1])
    assert np.array_equal(plane(lo, mrlbm.ZGHOST_ABOVE), m[:, hi.z0])
    assert np.array_equal(plane(hi, mrlbm.ZGHOST_BELOW), m[:, lo.z1 - 1])
    assert np.array_equal(plane(hi, mrlbm.ZGHOST_ABOVE), m[:, 0])
    zs.close()


def test_copy_rejects_mismatched_slabs():
    a = mrlbm.Domain(mrlbm.make_desc(16, 16, 8, tau=0.6))
    b = mrlbm.Domain(mrlbm.make_desc(24, 16, 8, tau=0.6))
    with pytest.raises(mrlbm.MrlbmError, match="slabs differ"):
        mrlbm.check(mrlbm.lib().mrlbm_zslab_copy(a.h, mrlbm.ZPLANE_LAST, b.h, mrlbm.ZGHOST_BELOW))
    with pytest.raises(mrlbm.MrlbmError, match="ghost plane"):
        mrlbm.check(mrlbm.lib().mrlbm_zslab_copy(a.h, mrlbm.ZPLANE_LAST, a.h, mrlbm.ZPLANE_FIRST))
    a.close()
    b.close()


def test_one_nccl_rank_on_torch_stream():
    """The distributed driver with one rank: the domain launches on a torch
    stream and the exchange is queued there, the periodic exchange is a self copy, and the FP64 sums
    go through an NCCL all-reduce."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        d = mrlbm.make_desc(48, 32, 24, lattice=mrlbm.D3Q19, tau=0.58)
        rho, u = _random_flow((24, 32, 48), 9)
        mono = mrlbm.Domain(d)
        mono.init_flow(rho, *u)
        mono.step(16)
        want, ws = mono.moments(), mono.sums()
        mono.close()
        zs = zslab.ZSlabDomain.distributed(d, exchange="torch")
        assert zs.slabs[0].dom.get_stream() == zs.stream.cuda_stream != 0
        zs.init_flow(rho, *u)
        zs.step(16)
        got = zs.moments()
        s = zs.sums()
        zs.close()
        assert np.array_equal(got, want)
        assert s["mass"] == pytest.approx(ws["mass"], rel=1e-12)
        assert s["fluid_nodes"] == ws["fluid_nodes"]
    finally:
        dist.destroy_process_group()



def test_one_rank_library_nccl_exchange():
    """The library's own NCCL driver (mrlbm_zslab_exchange_nccl), one rank:
    a single periodic slab is its own neighbour below and above, so each
    step's exchange is an NCCL send/receive to itself of both boundary
    planes; the result equals the undivided periodic domain bit for bit.
    Bootstrapped through torch.distributed (unique id broadcast) and, second,
    with no torch at all (mrlbm_nccl_unique_id / mrlbm_nccl_comm_init)."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    d = mrlbm.make_desc(48, 32, 24, lattice=mrlbm.D3Q27, tau=0.57)
    rho, u = _random_flow((24, 32, 48), 13)
    mono = mrlbm.Domain(d)
    mono.init_flow(rho, *u)
    mono.step(12)
    want = mono.moments()
    mono.close()

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        zs = zslab.ZSlabDomain.distributed(d)
        assert zs.comm is not None and zs.nccl_peers == (0, 0)
        zs.init_flow(rho, *u)
        zs.step(12)
        got = zs.moments()
        zs.close()
        assert np.array_equal(got, want)
    finally:
        dist.destroy_process_group()

    # no torch on any path: the id and the communicator from the library
    comm = mrlbm.NcclComm(1, mrlbm.nccl_unique_id(), 0)
    slab = mrlbm.Domain(zslab.slab_desc(d, 0, 24))
    slab.init_flow(rho, *u)
    L = mrlbm.lib()
    mrlbm.check(L.mrlbm_zslab_exchange_nccl(slab.h, comm.h, 0, 0))
    for _ in range(12):
        slab.step(1)
        mrlbm.check(L.mrlbm_zslab_exchange_nccl(slab.h, comm.h, 0, 0))
    got2 = slab.moments()
    slab.synchronize()
    slab.close()
    comm.close()
    assert np.array_equal(got2, want)


def test_outflow_channel_with_a_one_plane_top_slab():
    """Velocity inlet at z = 0 and an outflow face at z = nz - 1, cut into 7
    slabs whose top one is a single plane: its outflow nodes read their
    inward neighbour's previous-step moments from the ghost plane the slab
    below filled."""
    from test_gpu_parity import channel_node_types

    nx, ny, nz = 20, 18, 13
    assert zslab.slab_bounds(nz, 7)[-1] == (12, 13)
    d = mrlbm.make_desc(nx, ny, nz, lattice=mrlbm.D3Q19, periodic=(0, 0, 0), tau=0.7,
                        bc_velocity=[(0.0, 0.0, 0.03)])
    want, got, _ = _run_both(d, 7, 60, nt=channel_node_types(nx, ny, nz), init=lambda dom: dom.init_uniform())
    assert float(np.mean(want[3, -1, 1:-1, 1:-1])) > 0.0
    assert np.array_equal(got, want)


def test_power_law_cavity_omega_travels_with_the_planes():
    """Power-law fluid: omega is stored as moment 10 (six moment pairs, the
    last one padded) and the slabs' ghost planes carry it."""
    d = mrlbm.make_desc(30, 28, 26, lattice=mrlbm.D3Q19, periodic=(0, 0, 0), tau=0.6,
                        bc_velocity=[(0.05, 0.0, 0.0)] + [(0.0, 0.0, 0.0)] * 3,
                        rheology=mrlbm.POWERLAW, nnf_n=0.7)
    want, got, _ = _run_both(d, 3, 40, nt=mrlbm.lid_cavity_node_types(30, 28, 26, 1))
    assert want.shape[0] == 11
    assert np.array_equal(got, want)
