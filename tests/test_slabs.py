"""The z-slab decomposition's host logic on the CPU: the neighbour geometry (the z part of the
reference's grid_structure, parallel.f90:230-241), cutting and joining states, and the halo
exchange itself between gloo processes on 127.0.0.1 (world size 2 and 4, one or two slabs per
process, periodic and zero-gradient z), checked against the box's own wrapped planes; and the
min / sum reductions of the CFL step and the history."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dumses_hybrid_b200 import Params
from dumses_hybrid_b200.slabs import (LOWER, UPPER, HaloExchange, Neighbours, join_states, reduce_values,
                                      slab_params, split_state)


def test_neighbours_periodic_and_zero_gradient():
    nb = Neighbours(4, zero_gradient=False)
    assert [nb.lower(z) for z in range(4)] == [3, 0, 1, 2]
    assert [nb.upper(z) for z in range(4)] == [1, 2, 3, 0]
    assert all(nb.takes_halo(z, s) for z in range(4) for s in (LOWER, UPPER))
    zg = Neighbours(4, zero_gradient=True)
    assert not zg.takes_halo(0, LOWER) and zg.takes_halo(0, UPPER)
    assert not zg.takes_halo(3, UPPER) and zg.takes_halo(3, LOWER)
    assert not Neighbours(1, False).takes_halo(0, LOWER)


def test_slab_params_split_join():
    box = Params(ndim=3, nx=4, ny=5, nz=12, zmin=-1.0, zmax=2.0)
    p = slab_params(box, 3, 2)
    assert (p.nz, p.nzslice, p.zposition, p.zmin, p.zmax) == (4, 3, 2, -1.0, 2.0)
    with pytest.raises(ValueError):
        slab_params(box, 5, 0)
    with pytest.raises(ValueError):
        slab_params(box, 6, 0)  # 2 planes per slab: less than a halo
    u = np.asfortranarray(np.random.default_rng(0).random(box.shape))
    parts = split_state(u, box, 3)
    assert [q.shape for q in parts] == [(10, 11, 10, 11)] * 3
    assert np.array_equal(parts[1][:, :, :, :], u[:, :, 4:14, :])
    assert np.array_equal(join_states(parts, box), u)


class FakeSlab:
    """A slab of a periodic field: planes (nz + 6, m) along z, 3 ghost planes each side."""

    def __init__(self, planes: np.ndarray):
        self.u = planes
        self.nz = planes.shape[0] - 6

    def halo_pack(self, side, buf):
        src = self.u[3:6] if side == LOWER else self.u[self.nz:self.nz + 3]
        buf.numpy()[:] = src.reshape(-1)

    def halo_unpack(self, side, buf):
        dst = self.u[0:3] if side == LOWER else self.u[self.nz + 3:self.nz + 6]
        dst[...] = buf.numpy().reshape(dst.shape)

    def sync(self):
        pass


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


NZ_SLAB, M = 4, 6  # planes per slab, values per plane


def box_planes(nzslice: int) -> np.ndarray:
    return np.arange(nzslice * NZ_SLAB * M, dtype=np.float64).reshape(nzslice * NZ_SLAB, M) + 1.0


def _rank_main(rank, world, per, zg, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = world * per
        box = box_planes(n)
        slabs = []
        for s in range(per):
            z = rank * per + s
            planes = np.full((NZ_SLAB + 6, M), -1.0)  # ghosts marked
            planes[3:3 + NZ_SLAB] = box[z * NZ_SLAB:(z + 1) * NZ_SLAB]
            slabs.append(FakeSlab(planes))
        make = lambda c: torch.zeros(c, dtype=torch.float64)  # noqa: E731
        ex = HaloExchange(slabs, rank * per, Neighbours(n, zg), 3 * M, make, dist)
        ex.exchange()
        dt = reduce_values(np.array([0.5 + rank]), "min", dist)
        tot = reduce_values(np.array([1.0 + rank, 2.0]), "sum", dist)
        q.put((rank, [s.u.copy() for s in slabs], float(dt[0]), tot.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,per,zg", [(2, 1, False), (2, 1, True), (4, 1, False), (2, 2, False), (2, 2, True)])
def test_gloo_halo_exchange_fills_ghosts_like_the_box(world, per, zg):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, per, zg, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict((r, (u, dt, tot)) for r, u, dt, tot in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    n = world * per
    box = box_planes(n)
    padded = np.pad(box, ((3, 3), (0, 0)), mode="wrap")
    for r in range(world):
        u, dt, tot = got[r]
        assert dt == 0.5 and tot == [sum(1.0 + k for k in range(world)), 2.0 * world]
        for s in range(per):
            z = r * per + s
            want = padded[z * NZ_SLAB:z * NZ_SLAB + NZ_SLAB + 6].copy()
            if zg and z == 0:
                want[:3] = -1.0  # the bottom slab fills its own lower ghosts; no halo arrives
            if zg and z == n - 1:
                want[-3:] = -1.0
            assert np.array_equal(u[s], want), (r, s)
