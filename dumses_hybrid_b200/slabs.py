"""z-slab decomposition of the MHD step over several contexts and processes.

The reference decomposes its box over MPI ranks (src/subroutines/parallel.f90:197-697): a
rank owns nx*ny*nz cells (nz = nzglob/nzslice, init.f90:190-197), finds its neighbours from
its position (grid_structure, parallel.f90:197-257), exchanges 3-deep ghost slabs of uin
after every boundary call (boundary_z, with MPI_Sendrecv or ncclSend/ncclRecv), takes the
box's CFL step with MPI_Allreduce(MIN) (physics.f90:123-129) and reduces the history sums
over the ranks (src/problem/mri/history.f90:176-245).

Here the box is split in z only: x keeps the shear-periodic boundary inside every slab and
FARGO needs whole y lines.  Each slab is a library context (`Params.nzslice`,
`Params.zposition`); a process holds one or more consecutive slabs (one per GPU in
production, several on one GPU in the tests); halos move between the slabs of a process as
device copies and between processes with `torch.distributed` point-to-point operations (NCCL
over NVLink on GPUs, gloo on CPUs).  The step is the reference's loop body with the exchange
where its boundary routine does it:

    dt = min over slabs of compute_dt          (all_reduce MIN over processes)
    godunov; fargo_update; boundary + halo exchange
    [dissipation + halo exchange]              (nu > 0 or eta > 0)

In FP64 the slabs together are bit-identical to the undecomposed box: every cell sees the same
neighbour values and the CFL minimum is exact.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from . import Context, Params

# sides of a slab
LOWER, UPPER = 0, 1


def slab_params(box: Params, nzslice: int, zposition: int) -> Params:
    """Parameters of slab `zposition` of a box split into `nzslice` z slabs (box.nz cells in z)."""
    if box.ndim != 3:
        raise ValueError("a z-slab decomposition needs ndim = 3")
    if nzslice < 1 or box.nz % nzslice:
        raise ValueError(f"nz = {box.nz} is not a multiple of nzslice = {nzslice}")
    if box.nz // nzslice < 3:
        raise ValueError("every slab needs at least 3 planes (its halo)")
    if nzslice == 1:
        return replace(box, nzslice=1, zposition=0)
    return replace(box, nz=box.nz // nzslice, nzslice=nzslice, zposition=zposition)


def split_state(u: np.ndarray, box: Params, nzslice: int) -> list[np.ndarray]:
    """The reference-layout state of the box cut into the slabs' states (each with its 3 ghost
    planes taken from the box's own array)."""
    nz = box.nz // nzslice
    return [np.asfortranarray(u[:, :, z * nz:z * nz + nz + 6, :]) for z in range(nzslice)]


def join_states(parts: list[np.ndarray], box: Params) -> np.ndarray:
    """The box's state from its slabs in z order (active planes from each slab, the box's
    lower/upper ghost planes from the first/last slab)."""
    nz = box.nz // len(parts)
    u = np.zeros(box.shape, order="F")
    for z, p in enumerate(parts):
        u[:, :, 3 + z * nz:3 + (z + 1) * nz, :] = p[:, :, 3:3 + nz, :]
    u[:, :, :3, :] = parts[0][:, :, :3, :]
    u[:, :, -3:, :] = parts[-1][:, :, -3:, :]
    return u


class Neighbours:
    """The z part of grid_structure (parallel.f90:230-241): the lower and upper slab of a
    position, periodic in z; with a zero-gradient z boundary the bottom and top slabs fill
    their outer ghost planes themselves and take no halo there."""

    def __init__(self, nzslice: int, zero_gradient: bool):
        self.n = nzslice
        self.zg = zero_gradient

    def lower(self, z: int) -> int:
        return (z - 1) % self.n

    def upper(self, z: int) -> int:
        return (z + 1) % self.n

    def takes_halo(self, z: int, side: int) -> bool:
        """Whether slab z fills its `side` ghost planes from a neighbour's halo."""
        if self.n == 1:
            return False  # one slab fills its own z ghosts (periodic or zero-gradient)
        return not (self.zg and ((side == LOWER and z == 0) or (side == UPPER and z == self.n - 1)))


class HaloExchange:
    """Moves the halos of the slabs that one process holds (consecutive positions
    first .. first + len(slabs) - 1) to their neighbours, locally or through a process group.

    A slab is any object with `halo_pack(side, buf)`, `halo_unpack(side, buf)` and `sync()`,
    where `buf` is a 1-D float64 torch tensor of `count` elements (device memory for library
    contexts, host memory for gloo)."""

    def __init__(self, slabs, first: int, neighbours: Neighbours, count: int, make_buffer, dist=None, group=None):
        self.slabs = list(slabs)
        self.first = first
        self.nb = neighbours
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group) if dist is not None else 0
        self.world = dist.get_world_size(group) if dist is not None else 1
        if len(self.slabs) * self.world != neighbours.n:
            raise ValueError("every process must hold the same number of slabs, nzslice in all")
        self.send = [[make_buffer(count), make_buffer(count)] for _ in self.slabs]
        self.recv = [make_buffer(count), make_buffer(count)]  # from the lower / upper process

    def _local(self, z: int) -> int | None:
        s = z - self.first
        return s if 0 <= s < len(self.slabs) else None

    def exchange(self) -> None:
        nb = self.nb
        zs = [self.first + s for s in range(len(self.slabs))]
        # pack every side a neighbour takes: my lower planes go to my lower neighbour's upper side
        for s, z in enumerate(zs):
            if nb.takes_halo(nb.lower(z), UPPER):
                self.slabs[s].halo_pack(LOWER, self.send[s][LOWER])
            if nb.takes_halo(nb.upper(z), LOWER):
                self.slabs[s].halo_pack(UPPER, self.send[s][UPPER])
        for sl in self.slabs:
            sl.sync()
        # across processes: the bottom slab talks to the process below, the top slab to the one
        # above, in one fixed order on every process (sends to the lower and upper process,
        # then receives from the upper and lower one), so that with two processes, where both
        # neighbours are the same process, the n-th send meets the n-th receive
        if self.world > 1:
            prev, nxt = (self.rank - 1) % self.world, (self.rank + 1) % self.world
            zb, zt = zs[0], zs[-1]
            P2P, d = self.dist.P2POp, self.dist
            ops = []
            if nb.takes_halo(nb.lower(zb), UPPER) and self._local(nb.lower(zb)) is None:
                ops.append(P2P(d.isend, self.send[0][LOWER], prev, self.group))
            if nb.takes_halo(nb.upper(zt), LOWER) and self._local(nb.upper(zt)) is None:
                ops.append(P2P(d.isend, self.send[-1][UPPER], nxt, self.group))
            if nb.takes_halo(zt, UPPER) and self._local(nb.upper(zt)) is None:
                ops.append(P2P(d.irecv, self.recv[UPPER], nxt, self.group))
            if nb.takes_halo(zb, LOWER) and self._local(nb.lower(zb)) is None:
                ops.append(P2P(d.irecv, self.recv[LOWER], prev, self.group))
            if ops:
                for w in d.batch_isend_irecv(ops):
                    w.wait()
        # unpack: from a local neighbour's send buffer, or from what another process sent
        for s, z in enumerate(zs):
            for side, other in ((LOWER, nb.lower(z)), (UPPER, nb.upper(z))):
                if not nb.takes_halo(z, side):
                    continue
                o = self._local(other)
                buf = self.send[o][1 - side] if o is not None else self.recv[side]
                self.slabs[s].halo_unpack(side, buf)


def reduce_values(values: np.ndarray, op: str, dist=None, group=None, device="cpu") -> np.ndarray:
    """all_reduce of a small FP64 vector over the processes ("min" or "sum"); the identity
    without a process group."""
    if dist is None:
        return np.asarray(values, dtype=np.float64)
    import torch
    t = torch.tensor(np.asarray(values, dtype=np.float64), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN if op == "min" else dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


class _ContextSlab:
    """A library context seen through the HaloExchange interface."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def halo_pack(self, side, buf):
        self.ctx.halo_pack(side, buf.data_ptr())

    def halo_unpack(self, side, buf):
        self.ctx.halo_unpack(side, buf.data_ptr())

    def sync(self):
        self.ctx.sync()


class SlabSet:
    """The slabs of a decomposed box that this process holds, stepped like one box.

    box      the whole box (nz = all z cells)
    nzslice  slabs in all
    dist     torch.distributed when the slabs are spread over processes (each holds
             nzslice / world consecutive slabs), else None (this process holds them all)
    device   CUDA device of this process's contexts and halo buffers"""

    def __init__(self, box: Params, nzslice: int, dist=None, group=None, device: int = 0):
        import torch
        self.box = box
        self.nzslice = nzslice
        self.dist = dist
        self.group = group
        world = dist.get_world_size(group) if dist is not None else 1
        rank = dist.get_rank(group) if dist is not None else 0
        if nzslice % world:
            raise ValueError("nzslice must be a multiple of the number of processes")
        per = nzslice // world
        self.first = rank * per
        self.params = [replace(slab_params(box, nzslice, z), device=device) for z in range(self.first, self.first + per)]
        self.ctxs = [Context(p) for p in self.params]
        self.device = device
        self.torch_device = torch.device("cuda", device)
        self._allreduce_device = self.torch_device
        if dist is not None and dist.get_backend(group) == "gloo":
            self._allreduce_device = torch.device("cpu")
        self.rebuild_exchange()

    def rebuild_exchange(self) -> None:
        """Set up the halo exchange of the current contexts (after replacing them)."""
        import torch
        count = self.ctxs[0].halo_count
        make = lambda n: torch.empty(n, dtype=torch.float64, device=self.torch_device)  # noqa: E731
        self.halo = HaloExchange([_ContextSlab(c) for c in self.ctxs], self.first,
                                 Neighbours(self.nzslice, self.box.bdtypez == "zero_gradient"), count, make,
                                 self.dist, self.group)

    # ---- the reference's routines over the slabs ----
    def upload(self, parts: list[np.ndarray]) -> None:
        """States of this process's slabs (from split_state)."""
        for c, u in zip(self.ctxs, parts):
            c.upload(u)

    def download(self) -> list[np.ndarray]:
        return [c.download() for c in self.ctxs]

    def _reduce(self, values: np.ndarray, op: str) -> np.ndarray:
        return reduce_values(values, op, self.dist, self.group, self._allreduce_device)

    def compute_dt(self) -> float:
        """The box's CFL step: the minimum over the slabs (physics.f90:123-129)."""
        dt = min(c.compute_dt() for c in self.ctxs)
        return float(self._reduce(np.array([dt]), "min")[0])

    def boundary(self, time: float, dt: float) -> None:
        for c in self.ctxs:
            c.boundary(time, dt)
        self.halo.exchange()

    def godunov(self, dt: float, time: float) -> None:
        for c in self.ctxs:
            c.godunov(dt, time)

    def fargo_update(self, dt: float) -> None:
        for c in self.ctxs:
            c.fargo_update(dt)

    def dissipation(self, time: float, dt: float) -> None:
        if self.box.nu > 0 or self.box.eta > 0:
            for c in self.ctxs:
                c.dissipation(time, dt)
            self.halo.exchange()

    def step(self, time: float) -> tuple[float, float]:
        """One pass of the loop body of dumses.f90:82-120; returns (time + dt, dt)."""
        dt = self.compute_dt()
        self.godunov(dt, time)
        if self.box.fargo:
            self.fargo_update(dt)
        self.boundary(time, dt)
        self.dissipation(time, dt)
        return time + dt, dt

    def history(self) -> np.ndarray:
        """The box's MRI history values (dg_history's order), reduced over the slabs as the
        reference's compute_yz_mean and vol_average do."""
        col = sum(c.history_columns() for c in self.ctxs)
        col = self._reduce(np.ascontiguousarray(col).reshape(-1), "sum").reshape(-1, 2)
        slab_nz = self.box.nz // self.nzslice
        colmean = col / self.box.ny / slab_nz / self.nzslice
        share = sum(c.history_share(colmean) for c in self.ctxs)
        return self._reduce(share, "sum")

    def sync(self) -> None:
        for c in self.ctxs:
            c.sync()

    def close(self) -> None:
        for c in self.ctxs:
            c.close()
        self.ctxs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
