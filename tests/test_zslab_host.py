"""Host logic of the z-slab decomposition on CPU: slab bounds, the pairing of
the exchange plan, and gloo runs of two and three ranks whose slabs are
stepped by the FP64 oracle (a test-side stand-in for the library domain)
through the same exchange code as the NCCL path (zslab.run_exchange), checked
against the undivided oracle domain: identical moments, bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

import mrlbm  # noqa: E402
import zslab  # noqa: E402


def test_slab_bounds():
    for nz in (1, 2, 7, 64, 257):
        for parts in range(1, min(nz, 9) + 1):
            b = zslab.slab_bounds(nz, parts)
            assert b[0][0] == 0 and b[-1][1] == nz
            assert all(b[i][1] == b[i + 1][0] for i in range(parts - 1))
            sizes = [z1 - z0 for z0, z1 in b]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        zslab.slab_bounds(4, 5)


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_exchange_plan_pairs(parts, periodic):
    """Matching the k-th send from a to b with the k-th receive at b from a
    (NCCL's rule for point-to-point operations between two ranks) delivers
    every boundary plane to the right ghost plane of the right neighbour."""
    plans = [zslab.exchange_plan(i, parts, periodic) for i in range(parts)]
    delivered = {}
    for a in range(parts):
        for b in range(parts):
            if a == b:
                continue
            sends = [(w, d) for op, p, w, d in plans[a] if op == "send" and p == b]
            recvs = [(w, d) for op, p, w, d in plans[b] if op == "recv" and p == a]
            assert len(sends) == len(recvs)
            for (sw, sd), (rw, rd) in zip(sends, recvs):
                assert sd == rd    # same direction tag (gloo matches on it)
                delivered[(b, rw)] = (a, sw)
    for i in range(parts):
        for op, p, w, d in plans[i]:
            if op == "copy":
                delivered[(i, zslab.GHOST_OF[d])] = (i, w)
    for i in range(parts):
        below, above = zslab.neighbours(i, parts, periodic)
        want = {}
        if below is not None:
            want[(i, mrlbm.ZGHOST_BELOW)] = (below, mrlbm.ZPLANE_LAST)
        if above is not None:
            want[(i, mrlbm.ZGHOST_ABOVE)] = (above, mrlbm.ZPLANE_FIRST)
        got = {k: v for k, v in delivered.items() if k[0] == i}
        assert got == want


class OracleSlab:
    """Slab [z0, z1) held by the oracle as a domain of z1 - z0 + 2 planes,
    periodic in z, whose outer planes are the ghost planes: solid nodes (the
    oracle keeps their moments through a step), holding the neighbours'
    planes after each exchange, or the exterior state at a non-periodic end
    (whose reconstruction is the oracle's exterior populations)."""

    def __init__(self, desc, nt, m0, z0, z1):
        import parity_util

        self.z0, self.z1 = z0, z1
        ext_desc = zslab.slab_desc(desc, z0, z1)
        ext_desc.nz = z1 - z0 + 2
        ext_desc.periodic[2] = 1
        nte = np.full((z1 - z0 + 2,) + nt.shape[1:], 0xFF, dtype=np.uint32)
        nte[1:-1] = nt[z0:z1]
        self.o = parity_util.oracle_for(ext_desc, nte)
        ext = np.zeros(self.o.nm)
        ext[:10] = np.array(self.o.desc.exterior[:10])
        if desc.thermal:
            ext[10] = desc.t_reference
        me = np.empty((z1 - z0 + 2,) + m0.shape[1:])
        me[1:-1] = m0[z0:z1]
        me[0] = me[-1] = ext
        self.o.set_moments(me)
        self.rx = {}

    def step(self, n=1):
        self.o.step(n)

    def _plane(self, which):
        return {mrlbm.ZPLANE_FIRST: 1, mrlbm.ZPLANE_LAST: -2, mrlbm.ZGHOST_BELOW: 0, mrlbm.ZGHOST_ABOVE: -1}[which]

    def send_buffers(self, which):
        import torch

        return [torch.from_numpy(np.ascontiguousarray(self.o.moments()[self._plane(which)]).reshape(-1))]

    def recv_buffers(self, which):
        import torch

        t = torch.empty(int(np.prod(self.o.moments().shape[1:])), dtype=torch.float64)
        self.rx[which] = t
        return [t]

    def recv_done(self):
        if not self.rx:
            return
        m = self.o.moments()
        for which, t in self.rx.items():
            m[self._plane(which)] = t.numpy().reshape(m.shape[1:])
        self.o.set_moments(m)
        self.rx = {}

    def local_copy(self, src_which, dst_which):
        m = self.o.moments()
        m[self._plane(dst_which)] = m[self._plane(src_which)]
        self.o.set_moments(m)

    def interior(self):
        return self.o.moments()[1:-1]


def _case(name):
    """(library descriptor, node types (nz, ny, nx), initial oracle moments
    (nz, ny, nx, nm), steps) of a small case."""
    import parity_util

    rng = np.random.default_rng(7)
    if name == "tgv_q27":
        d = mrlbm.make_desc(12, 10, 9, lattice=mrlbm.D3Q27, tau=0.56)
        nt = np.zeros((9, 10, 12), dtype=np.uint32)
        steps = 6
    elif name == "cavity_q19":
        d = mrlbm.make_desc(10, 11, 9, lattice=mrlbm.D3Q19, periodic=(0, 0, 0), tau=0.6,
                            bc_velocity=[(0.05, 0, 0)] + [(0, 0, 0)] * 3)
        nt = mrlbm.lid_cavity_node_types(10, 11, 9, 1).reshape(9, 11, 10)
        steps = 8
    else:   # thermal Rayleigh-Benard slab: plates at z = 0 and z = nz - 1
        th = dict(diffusivity=0.02, reference=1.0, gravity_beta=(0.0, 0.0, 1e-3), wall=(1.5, 0.5, 1.0, 1.0))
        d = mrlbm.make_desc(8, 8, 10, lattice=mrlbm.D3Q19, periodic=(1, 1, 0), tau=0.55, thermal=th)
        nt = np.zeros((10, 8, 8), dtype=np.uint32)
        nt[0] = mrlbm.BACK | mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET) | mrlbm.THERMAL_INDEX(0)
        nt[-1] = mrlbm.FRONT | mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET) | mrlbm.THERMAL_INDEX(1)
        steps = 6
    shape = (d.nz, d.ny, d.nx)
    mono = parity_util.oracle_for(d, nt)
    rho = 1.0 + 0.01 * rng.standard_normal(shape)
    u = [0.02 * rng.standard_normal(shape) for _ in range(3)]
    mono.init_from_macro(rho, *u)
    m0 = mono.moments()
    if d.thermal:
        m0[..., 10] += 0.1 * rng.standard_normal(shape)
    return d, nt, m0, steps


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, name, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "mr-lbm_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import zslab as zs

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d, nt, m0, steps = _case(name)
        z0, z1 = zs.slab_bounds(d.nz, world)[rank]
        slab = OracleSlab(d, nt, m0, z0, z1)
        periodic_z = bool(d.periodic[2])
        zs.run_exchange(slab, rank, world, periodic_z)
        for _ in range(steps):
            slab.step(1)
            zs.run_exchange(slab, rank, world, periodic_z)
        q.put((rank, z0, z1, slab.interior()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("tgv_q27", 2), ("tgv_q27", 3), ("cavity_q19", 3),
                                        ("thermal_rb", 2), ("tgv_q27", 1)])
def test_gloo_slabs_match_undivided_oracle(name, world):
    import parity_util
    import torch.multiprocessing as mp

    d, nt, m0, steps = _case(name)
    mono = parity_util.oracle_for(d, nt)
    mono.set_moments(m0)
    mono.step(steps)
    want = mono.moments()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.all(np.isfinite(want))
    got = np.concatenate([m for _, _, _, m in out], axis=0)
    assert [(z0, z1) for _, z0, z1, _ in out] == zslab.slab_bounds(d.nz, world)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
