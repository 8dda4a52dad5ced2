"""One grid split into z-slabs: several GPUs (or several handles on one GPU) advance one grid.

Decomposition.  The Nz planes are split into `parts` contiguous owned ranges.  Each part is an
ordinary grid (a Simulation) over its owned planes plus halo planes on every side that has a
neighbour: `halo` below and `halo` + 1 above.  A launch of b <= halo steps (the tiled kernel's
BLT) leaves the owned planes exact.  The kernel holds a grid's first and last planes fixed, so a
slab's own outer planes go wrong from the first step, and the error moves in one plane per
step: E at plane p reads H at p and p-1, H at p reads E at p and p+1.  From the bottom plane, E
and H are wrong on planes 0 .. b-1 after b steps; from the top plane P, H is wrong down to
P - b (one plane further, because the top plane's E is never updated and H^1(P-1) reads it).
After every launch each part sends its `halo` + 1 lowest owned planes of all six components down
and its `halo` highest owned planes up, into the neighbours' halos: one exchange step per
temporal block, (2 * halo + 1) * Nx * Ny * 6 values per interior face.  The global first and
last planes are the first and last planes of the end parts, so the reference's fixed outer
faces are kept.

Inputs follow the planes: coefficients are sliced from the global arrays (a slab's pseudo-PML
grading must be the global grid's, so they are not rebuilt per slab); a source goes to every
part whose local planes (owned or halo) contain it, because a halo plane's updates feed the
owned planes within the block; a DFT monitor lives on the part that owns its plane.

HaloPlan is the index arithmetic (no GPU); ZSlabGrid runs all parts in one process (one or
several devices); exchange_dist() is the same exchange between processes over
torch.distributed (NCCL for device buffers; the tests run it over gloo).  No reference
counterpart: gDiamond runs one grid on one GPU.
"""
from __future__ import annotations

import numpy as np

from . import COMPONENTS, Simulation


class HaloPlan:
    """Owned and local z-ranges of each part, and the planes each exchange moves."""

    def __init__(self, nz, parts, halo):
        nz, parts, halo = int(nz), int(parts), int(halo)
        if parts < 1 or halo < 1:
            raise ValueError("parts and halo must be positive")
        base, extra = divmod(nz, parts)
        if base < halo + 1 or (parts == 1 and nz < 3):
            raise ValueError(f"{nz} planes cannot be split into {parts} parts of >= {halo + 1} "
                             "planes")
        self.nz, self.parts, self.halo = nz, parts, halo
        self.own, self.loc = [], []
        z = 0
        for r in range(parts):
            n = base + (1 if r < extra else 0)
            self.own.append((z, z + n))
            lo = z - halo if r > 0 else 0
            hi = z + n + halo + 1 if r < parts - 1 else nz
            self.loc.append((lo, hi))
            z += n

    def local_nz(self, r):
        lo, hi = self.loc[r]
        return hi - lo

    def to_local(self, r, k):
        """Local plane index of global plane k on part r, or None when k is not stored there."""
        lo, hi = self.loc[r]
        return k - lo if lo <= k < hi else None

    def owner(self, k):
        for r, (lo, hi) in enumerate(self.own):
            if lo <= k < hi:
                return r
        raise ValueError(f"plane {k} outside the grid")

    def sends(self, r):
        """[(peer, first global plane, planes)] part r sends after a block."""
        lo, hi = self.own[r]
        out = []
        if r > 0:
            out.append((r - 1, lo, self.halo + 1))
        if r < self.parts - 1:
            out.append((r + 1, hi - self.halo, self.halo))
        return out

    def recvs(self, r):
        """[(peer, first global plane, planes)] part r receives into its halos."""
        lo, hi = self.own[r]
        out = []
        if r > 0:
            out.append((r - 1, lo - self.halo, self.halo))
        if r < self.parts - 1:
            out.append((r + 1, hi, self.halo + 1))
        return out


def slice_planes(arr, shape, lo, hi):
    """Planes [lo, hi) of a flat x-fastest array of shape (nx, ny, nz)."""
    nx, ny, nz = shape
    return np.ascontiguousarray(np.asarray(arr).reshape(nz, ny, nx)[lo:hi]).reshape(-1)


def localize_sources(plan, r, sources):
    """The sources part r must apply (global source dicts -> local copies)."""
    out = []
    for s in sources:
        k = plan.to_local(r, int(s["k"]))
        if k is not None:
            d = dict(s)
            d["k"] = k
            out.append(d)
    return out


def _block_bytes(esz, nk, ny, nx):
    """Bytes of nk planes of all six components; esz: bytes per value of each component."""
    return sum(int(e) * nk * ny * nx for e in esz)


def _block(sim, k0, nk, esz, device, stream):
    """Flat uint8 tensor of planes [k0, k0+nk) (local) of the six components in their raw
    storage format, one component after another (components may differ in size: f16e)."""
    import torch
    nx, ny, _ = sim.shape
    buf = torch.empty(_block_bytes(esz, nk, ny, nx), dtype=torch.uint8, device=device)
    off = 0
    for c in range(6):
        sim.get_planes_device(c, k0, nk, buf.data_ptr() + off, stream)
        off += int(esz[c]) * nk * ny * nx
    return buf


def _unblock(sim, k0, nk, buf, esz, stream):
    nx, ny, _ = sim.shape
    off = 0
    for c in range(6):
        sim.set_planes_device(c, k0, nk, buf.data_ptr() + off, stream)
        off += int(esz[c]) * nk * ny * nx


class ZSlabGrid:
    """A grid of nx x ny x nz cells run as `parts` z-slabs in this process.

    devices: one CUDA ordinal per part (default: all on device 0).  Every part runs the tiled
    kernel with BLT = halo; step(T) advances in blocks of `halo` steps with an exchange after
    each block.  Results are read back per global component and monitor.
    """

    def __init__(self, nx, ny, nz, parts, halo=2, devices=None, storage="f32", tile_rows=0,
                 kernel="tiled"):
        self.shape = (int(nx), int(ny), int(nz))
        self.plan = HaloPlan(nz, parts, halo)
        self.devices = list(devices) if devices is not None else [0] * parts
        self.sims = [Simulation(nx, ny, self.plan.local_nz(r), device=self.devices[r],
                                kernel=kernel, blt=halo, tile_rows=tile_rows, storage=storage)
                     for r in range(parts)]
        self.esz = [self.sims[0].component_bytes(c) for c in range(6)]
        self.monitors = []  # global id -> (part, local id)
        self.t = 0

    def set_coefficients(self, coef12):
        for r, sim in enumerate(self.sims):
            lo, hi = self.plan.loc[r]
            sim.set_coefficients([slice_planes(c, self.shape, lo, hi) for c in coef12])

    def set_sources(self, sources):
        for r, sim in enumerate(self.sims):
            sim.set_sources(localize_sources(self.plan, r, list(sources)))

    def add_dft_monitor(self, component, k, freqs, scale=1.0, dt=np.float32(0.05)):
        r = self.plan.owner(int(k))
        mid = self.sims[r].add_dft_monitor(component, self.plan.to_local(r, int(k)), freqs,
                                           scale, dt)
        self.monitors.append((r, mid))
        return len(self.monitors) - 1

    def reset(self):
        for sim in self.sims:
            sim.reset()
        self.t = 0

    def exchange(self):
        """Halo exchange after a block (every part's current field set)."""
        import torch
        for sim in self.sims:
            sim.sync()
        for r, sim in enumerate(self.sims):
            lo = self.plan.loc[r][0]
            for peer, k0, nk in self.plan.sends(r):
                dev = f"cuda:{self.devices[r]}"
                with torch.cuda.device(self.devices[r]):
                    buf = _block(sim, k0 - lo, nk, self.esz, dev, None)
                    sim.sync()
                dst = self.sims[peer]
                with torch.cuda.device(self.devices[peer]):
                    buf = buf.to(f"cuda:{self.devices[peer]}")
                    torch.cuda.synchronize(self.devices[peer])
                    _unblock(dst, k0 - self.plan.loc[peer][0], nk, buf, self.esz, None)
                    dst.sync()

    def step(self, T):
        T = int(T)
        done = 0
        while done < T:
            b = min(self.plan.halo, T - done)
            for sim in self.sims:
                sim.step(b)
            if self.plan.parts > 1:
                self.exchange()
            done += b
        self.t += T

    def sync(self):
        for sim in self.sims:
            sim.sync()

    def get_field(self, component):
        """The global component (flat, x-fastest) assembled from the owned planes."""
        nx, ny, nz = self.shape
        out = np.empty((nz, ny, nx), np.float32)
        for r, sim in enumerate(self.sims):
            lo, hi = self.plan.own[r]
            l0 = lo - self.plan.loc[r][0]
            f = sim.get_field(component).reshape(-1, ny, nx)
            out[lo:hi] = f[l0:l0 + hi - lo]
        return out.reshape(-1)

    def fields(self):
        return [self.get_field(c) for c in COMPONENTS]

    def get_dft(self, monitor_id):
        r, mid = self.monitors[monitor_id]
        return self.sims[r].get_dft(mid)

    def close(self):
        for sim in self.sims:
            sim.close()
        self.sims = []


def exchange_dist(plan, rank, get_block, put_block, make_buffer):
    """The halo exchange of part `rank` with its neighbours over torch.distributed.

    get_block(k0, nk) -> tensor of the planes to send (global plane k0 on); put_block(k0, nk,
    tensor) stores received planes; make_buffer(nk) -> an empty receive tensor.  Sends and
    receives are posted together (isend / irecv) so neighbours cannot deadlock; every rank of
    the group calls this after every block, in the same order.
    """
    import torch.distributed as dist
    reqs, recvs = [], []
    for peer, k0, nk in plan.recvs(rank):
        buf = make_buffer(nk)
        reqs.append(dist.irecv(buf, src=peer))
        recvs.append((k0, nk, buf))
    sends = []
    for peer, k0, nk in plan.sends(rank):
        buf = get_block(k0, nk)
        sends.append(buf)  # kept alive until the send completes
        reqs.append(dist.isend(buf, dst=peer))
    for q in reqs:
        q.wait()
    for k0, nk, buf in recvs:
        put_block(k0, nk, buf)


class DistZSlab:
    """This process's part of a grid split over the ranks of the default torch.distributed group
    (one rank per GPU; NCCL moves the halo planes over NVLink between device buffers).

    Every rank constructs it with the same global arguments and calls the same methods in the
    same order; step(T) runs blocks of `halo` steps, each followed by exchange_dist().
    """

    def __init__(self, nx, ny, nz, halo=2, device=None, storage="f32", tile_rows=0,
                 kernel="tiled"):
        import torch
        import torch.distributed as dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.shape = (int(nx), int(ny), int(nz))
        self.plan = HaloPlan(nz, self.world, halo)
        self.lo = self.plan.loc[self.rank][0]
        self.sim = Simulation(nx, ny, self.plan.local_nz(self.rank), device=self.device,
                              kernel=kernel, blt=halo, tile_rows=tile_rows, storage=storage)
        self.esz = [self.sim.component_bytes(c) for c in range(6)]
        self.monitors = []
        self.t = 0
        # One stream for the slab's kernels, its halo copies and NCCL, so the sends read planes
        # that are complete and the received planes land before the next launch.  (torch's
        # default stream would reach the C-ABI as NULL, i.e. the handle's own stream, which
        # NCCL does not wait for.)
        self.stream = torch.cuda.Stream(self.device)

    def set_coefficients(self, coef12):
        lo, hi = self.plan.loc[self.rank]
        self.sim.set_coefficients([slice_planes(c, self.shape, lo, hi) for c in coef12])

    def set_sources(self, sources):
        self.sim.set_sources(localize_sources(self.plan, self.rank, list(sources)))

    def add_dft_monitor(self, component, k, freqs, scale=1.0, dt=np.float32(0.05)):
        """Registers the monitor on its owner; returns (owner rank, id on the owner)."""
        r = self.plan.owner(int(k))
        mid = None
        if r == self.rank:
            mid = self.sim.add_dft_monitor(component, self.plan.to_local(r, int(k)), freqs,
                                           scale, dt)
        self.monitors.append((r, mid))
        return len(self.monitors) - 1

    def exchange(self):
        import torch
        nx, ny, _ = self.shape
        dev = f"cuda:{self.device}"
        stream = self.stream

        def get_block(k0, nk):
            return _block(self.sim, k0 - self.lo, nk, self.esz, dev, stream)

        def put_block(k0, nk, buf):
            _unblock(self.sim, k0 - self.lo, nk, buf, self.esz, stream)

        def make_buffer(nk):
            return torch.empty(_block_bytes(self.esz, nk, ny, nx), dtype=torch.uint8, device=dev)

        with torch.cuda.stream(stream):
            exchange_dist(self.plan, self.rank, get_block, put_block, make_buffer)

    def step(self, T, stream=None):
        """T steps on the slab's stream (kernels, halo copies and NCCL all run on it), ordered
        after the work queued so far on `stream` (default: the current torch stream), which in
        turn waits for the steps."""
        import torch
        caller = torch.cuda.current_stream(self.device) if stream is None else stream
        self.stream.wait_stream(caller)
        done = 0
        while done < int(T):
            b = min(self.plan.halo, int(T) - done)
            self.sim.step(b, self.stream)
            if self.world > 1:
                self.exchange()
            done += b
        caller.wait_stream(self.stream)
        self.t += int(T)

    def owned_field(self, component):
        """This rank's owned planes of a component ([planes][ny][nx] float32)."""
        nx, ny, _ = self.shape
        lo, hi = self.plan.own[self.rank]
        f = self.sim.get_field(component).reshape(-1, ny, nx)
        return f[lo - self.lo:hi - self.lo]

    def close(self):
        self.sim.close()
