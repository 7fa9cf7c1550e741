"""Z-slab decomposition of one MR-LBM domain (one slab per GPU, or several on
one GPU).

The reference runs one domain on one GPU (README.md:38; NZ_TOTAL == NZ in
every case, e.g. src/cases/benchmark/constants.inc:9).  A domain too large for
one GPU is cut here into slabs of whole z planes.  Each slab is an ordinary
domain of the library, non-periodic in z, and the only exchange of a time step
is its two z ghost planes: after every step the slab below sends its last
interior plane up and the slab above sends its first interior plane down, into
the receiver's own ghost planes, which its next step reads locally (the part
the reference's Z_0 / Z_1 ghost faces play between its thread blocks,
src/globalStructs.h ghostInterfaceData).  No kernel reads another GPU's memory.

Two drivers share the plan of the exchange:

* ``ZSlabDomain.local(desc, parts)`` keeps every slab in this process and
  moves planes with device copies (``mrlbm_zslab_copy``), each slab on its own
  stream with event ordering;
* ``ZSlabDomain.distributed(desc)`` owns the slab of this rank of
  torch.distributed (one process per GPU, NCCL over NVLink).  With an NCCL
  process group the exchange is the library's own (mrlbm_zslab_exchange_nccl:
  NCCL point-to-point operations in place, one group per step, queued on the
  domain's stream, so nothing waits on the host between steps and no PyTorch
  is on the data path; torch.distributed only hands the NCCL unique id to the
  ranks).  ``exchange="torch"`` (and any non-NCCL group, e.g. gloo) sends the
  planes as torch tensors viewing the library's buffers instead.

Arrays are numpy, x fastest, global shapes (nz, ny, nx) and (nm, nz, ny, nx)
as in ``mrlbm``.
"""
import numpy as np

import mrlbm

UP, DOWN = 0, 1   # direction tags of the two plane streams


def slab_bounds(nz, parts):
    """[z0, z1) of each of `parts` slabs: whole planes, sizes differing by at
    most one, the larger ones first."""
    if parts < 1 or parts > nz:
        raise ValueError("cannot cut %d planes into %d slabs" % (nz, parts))
    base, extra = divmod(nz, parts)
    out, z = [], 0
    for i in range(parts):
        n = base + (1 if i < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def neighbours(i, parts, periodic_z):
    """(below, above) slab indices of slab i; None at a non-periodic end."""
    below = i - 1 if i > 0 else (parts - 1 if periodic_z else None)
    above = i + 1 if i < parts - 1 else (0 if periodic_z else None)
    return below, above


def exchange_plan(i, parts, periodic_z):
    """Ordered operations of slab i for one exchange, as (op, peer, plane,
    direction) with op "send", "recv" or "copy" (peer is slab i itself: a
    local copy from `plane` to the ghost plane named by direction).

    Every slab lists the upward stream (its last plane to the slab above,
    which receives it as its ghost below) before the downward one (its first
    plane to the slab below, received as the ghost above), so the k-th send
    from a to b meets the k-th receive at b from a, also when a and b are
    each other's neighbours on both sides (two periodic slabs)."""
    below, above = neighbours(i, parts, periodic_z)
    ops = []
    if above == i:   # one periodic slab: its own neighbour on both sides
        return [("copy", i, mrlbm.ZPLANE_LAST, UP), ("copy", i, mrlbm.ZPLANE_FIRST, DOWN)]
    if above is not None:
        ops.append(("send", above, mrlbm.ZPLANE_LAST, UP))
    if below is not None:
        ops.append(("recv", below, mrlbm.ZGHOST_BELOW, UP))
    if below is not None:
        ops.append(("send", below, mrlbm.ZPLANE_FIRST, DOWN))
    if above is not None:
        ops.append(("recv", above, mrlbm.ZGHOST_ABOVE, DOWN))
    return ops


GHOST_OF = {UP: mrlbm.ZGHOST_BELOW, DOWN: mrlbm.ZGHOST_ABOVE}


def slab_desc(desc, z0, z1):
    """The descriptor of the slab [z0, z1) of `desc`: nz = z1 - z0, z not
    periodic (its ghost planes come from the neighbours)."""
    d = mrlbm.Desc.from_buffer_copy(desc)
    d.nz = z1 - z0
    d.periodic[2] = 0
    return d


class _DeviceBytes:
    """A device byte range as a __cuda_array_interface__ object (no stream
    semantics: the caller orders the access)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 2}


class GpuSlab:
    """One slab as a library domain; the plane buffers of the exchange are
    views of the domain's device memory (torch tensors, created per call since
    the planes move with the ping-pong parity)."""

    def __init__(self, desc, z0, z1):
        self.z0, self.z1 = z0, z1
        self.dom = mrlbm.Domain(slab_desc(desc, z0, z1))

    def step(self, n=1):
        self.dom.step(n)

    def _views(self, which):
        import torch

        p = self.dom.zplane(which)
        dev = torch.device("cuda", p["device"])
        return [torch.as_tensor(_DeviceBytes(p["base"] + k * p["pair_stride"], p["bytes"]), device=dev)
                for k in range(p["npairs"])]

    def send_buffers(self, which):
        return self._views(which)

    def recv_buffers(self, which):
        return self._views(which)

    def recv_done(self):
        pass

    def local_copy(self, src_which, dst_which):
        mrlbm.check(mrlbm.lib().mrlbm_zslab_copy(self.dom.h, src_which, self.dom.h, dst_which))

    def close(self):
        self.dom.close()


def run_exchange(slab, rank, parts, periodic_z, group=None):
    """One exchange of `slab` (slab index `rank` of `parts`) through
    torch.distributed point-to-point operations; returns the number of
    planes moved.  With NCCL the operations are queued after the work on the
    current stream and the current stream waits for them."""
    import torch.distributed as dist

    ops = []
    moved = 0
    for op, peer, which, direction in exchange_plan(rank, parts, periodic_z):
        if op == "copy":
            slab.local_copy(which, GHOST_OF[direction])
            moved += 1
            continue
        peer_rank = dist.get_global_rank(group, peer) if group is not None else peer
        bufs = slab.send_buffers(which) if op == "send" else slab.recv_buffers(which)
        fn = dist.isend if op == "send" else dist.irecv
        for k, t in enumerate(bufs):
            ops.append(dist.P2POp(fn, t, peer_rank, group, tag=direction * 64 + k))
        moved += op == "recv"
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    slab.recv_done()
    return moved


class ZSlabDomain:
    """One domain (descriptor `desc`, global sizes) cut into z slabs."""

    def __init__(self, desc, slabs, rank, parts, group, local):
        self.desc = desc
        self.slabs = slabs          # local: all slabs; distributed: this rank's
        self.rank, self.parts, self.group, self.local_mode = rank, parts, group, local
        self.periodic_z = bool(desc.periodic[2])
        self.bounds = slab_bounds(desc.nz, parts)
        self.nm = slabs[0].dom.nm
        self.shape = (desc.nz, desc.ny, desc.nx)

    @classmethod
    def local(cls, desc, parts):
        """All `parts` slabs in this process, on the current device."""
        slabs = [GpuSlab(desc, z0, z1) for z0, z1 in slab_bounds(desc.nz, parts)]
        return cls(desc, slabs, 0, parts, None, True)

    @classmethod
    def distributed(cls, desc, group=None, exchange="library"):
        """The slab of this rank of torch.distributed (initialised by the
        caller; one process per GPU with the device already selected).
        exchange="library" (NCCL groups): the library's NCCL driver on the
        domain's own stream, its communicator made from a unique id that rank
        0 broadcasts over the group.  exchange="torch" (and non-NCCL groups):
        the domain launches on a torch stream of its own (`.stream`) and the
        planes go as torch point-to-point operations queued on that stream."""
        import torch
        import torch.distributed as dist

        rank = dist.get_rank(group)
        parts = dist.get_world_size(group)
        z0, z1 = slab_bounds(desc.nz, parts)[rank]
        s = GpuSlab(desc, z0, z1)
        obj = cls(desc, [s], rank, parts, group, False)
        obj.comm = None
        if exchange == "library" and dist.get_backend(group) == "nccl":
            box = [mrlbm.nccl_unique_id() if rank == 0 else None]
            dist.broadcast_object_list(box, src=dist.get_global_rank(group, 0) if group is not None else 0,
                                       group=group)
            obj.comm = mrlbm.NcclComm(parts, box[0], rank)
            below, above = neighbours(rank, parts, obj.periodic_z)
            obj.nccl_peers = (-1 if below is None else below, -1 if above is None else above)
        else:
            stream = torch.cuda.Stream()
            s.dom.set_stream(stream.cuda_stream)
            obj.stream = stream
        return obj

    # -- setup (global arrays; each slab takes its planes)
    def set_node_types(self, nt):
        nt = np.asarray(nt, dtype=np.uint32).reshape(self.shape)
        for s in self.slabs:
            s.dom.set_node_types(nt[s.z0:s.z1])

    def init_flow(self, rho, ux, uy, uz):
        arrs = [np.asarray(a, dtype=np.float32).reshape(self.shape) for a in (rho, ux, uy, uz)]
        for s in self.slabs:
            s.dom.init_flow(*[a[s.z0:s.z1] for a in arrs])
        self.exchange()

    def init_uniform(self, u0=(0.0, 0.0, 0.0)):
        for s in self.slabs:
            s.dom.init_uniform(u0)
        self.exchange()

    def set_moments(self, m):
        m = np.asarray(m, dtype=np.float32).reshape((self.nm,) + self.shape)
        for s in self.slabs:
            s.dom.set_moments(np.ascontiguousarray(m[:, s.z0:s.z1]))
        self.exchange()

    # -- stepping
    def exchange(self):
        if self.local_mode:
            for i, s in enumerate(self.slabs):
                for op, peer, which, direction in exchange_plan(i, self.parts, self.periodic_z):
                    if op in ("send", "copy"):
                        dst = self.slabs[peer] if op == "send" else s
                        mrlbm.check(mrlbm.lib().mrlbm_zslab_copy(s.dom.h, which, dst.dom.h, GHOST_OF[direction]))
        elif self.comm is not None:
            below, above = self.nccl_peers
            mrlbm.check(mrlbm.lib().mrlbm_zslab_exchange_nccl(self.slabs[0].dom.h, self.comm.h, below, above))
        else:
            import torch

            with torch.cuda.stream(self.stream):
                run_exchange(self.slabs[0], self.rank, self.parts, self.periodic_z, self.group)

    def step(self, n=1):
        for _ in range(int(n)):
            for s in self.slabs:
                s.step(1)
            self.exchange()

    def synchronize(self):
        for s in self.slabs:
            s.dom.synchronize()

    # -- data
    def moments(self):
        """Local mode: the whole domain's moments.  Distributed mode: this
        rank's slab (planes self.slabs[0].z0 .. z1)."""
        if not self.local_mode:
            return self.slabs[0].dom.moments()
        return np.concatenate([s.dom.moments() for s in self.slabs], axis=1)

    def sums(self):
        """FP64 sums over the whole domain (mass, momentum, kinetic energy,
        fluid nodes, max speed, non-finite count)."""
        parts = [s.dom.sums() for s in self.slabs]
        v = np.array([[p["mass"], *p["momentum"], p["kinetic_energy"], p["fluid_nodes"], p["nonfinite"]]
                      for p in parts], dtype=np.float64).sum(axis=0)
        mx = max(p["max_speed"] for p in parts)
        if not self.local_mode:
            import torch
            import torch.distributed as dist

            dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
            t = torch.tensor(v, dtype=torch.float64, device=dev)
            dist.all_reduce(t, group=self.group)
            m = torch.tensor([mx], dtype=torch.float64, device=dev)
            dist.all_reduce(m, op=dist.ReduceOp.MAX, group=self.group)
            v, mx = t.cpu().numpy(), float(m.item())
        return {"mass": float(v[0]), "momentum": [float(x) for x in v[1:4]], "kinetic_energy": float(v[4]),
                "fluid_nodes": float(v[5]), "nonfinite": float(v[6]), "max_speed": mx}

    def close(self):
        for s in self.slabs:
            if not self.local_mode:
                s.dom.synchronize()
                s.dom.set_stream(None)
            s.close()
        self.slabs = []
        if getattr(self, "comm", None) is not None:
            self.comm.close()
            self.comm = None
