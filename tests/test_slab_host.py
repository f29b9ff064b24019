"""Slab decomposition host logic on CPU: row partitions, neighbours and ghost rows, and the
distributed transport's ghost-row exchange, wave-speed MAX and status agreement over real gloo
process groups (world size 2 and 3, walls and periodic y).  The slabs here are stand-ins that keep
their rows in CPU tensors tagged with the global row they came from; the device slabs run the same
transport code with NCCL."""
import contextlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dg_b200 import slab as S


@pytest.mark.parametrize("ny,nslabs,order,periodic", [
    (256, 2, 2, False), (256, 3, 2, False), (256, 4, 2, True), (64, 8, 2, False), (100, 3, 3, True),
    (90, 4, 1, False), (16, 2, 3, False), (40, 5, 2, True)])
def test_partition_covers_the_grid_with_tileable_slabs(ny, nslabs, order, periodic):
    rng = S.partition_rows(ny, nslabs, order, periodic)
    assert rng[0][0] == 0 and rng[-1][1] == ny
    assert all(a[1] == b[0] for a, b in zip(rng, rng[1:]))
    th = S.tile_rows(order)
    sizes = [r1 - r0 for r0, r1 in rng]
    assert min(sizes) >= S.GHOST
    assert max(sizes) - min(sizes) <= 2 * th + 1  # near-equal
    tileable = [(n + sum(S.ghost_rows(i, nslabs, periodic))) % th == 0 for i, n in enumerate(sizes)]
    if ny % th == 0:
        assert all(tileable), (rng, tileable)


def test_partition_rejects_too_many_slabs():
    with pytest.raises(ValueError):
        S.partition_rows(7, 4, 2, False)


def test_neighbours_and_ghost_rows():
    assert S.neighbours(0, 3, False) == (None, 1) and S.neighbours(2, 3, False) == (1, None)
    assert S.neighbours(0, 3, True) == (2, 1) and S.neighbours(2, 3, True) == (1, 0)
    assert S.neighbours(0, 2, True) == (1, 1)
    assert S.ghost_rows(0, 3, False) == (0, 2) and S.ghost_rows(1, 3, False) == (2, 2)
    assert S.ghost_rows(0, 1, True) == (0, 0)


def test_slab_problems_cover_their_rows():
    dec = S.Decomposition(2, 32, 24, 3, 0.0, 2.0, 0.0, 1.0, ("reflective", "transmissive") * 2, flux="rusanov",
                          limiter="m2l", cfl=0.3)
    hy = 1.0 / 24
    for i in range(3):
        prob, lo, hi, rows = dec.slab(i)
        r0, r1 = dec.ranges[i]
        assert prob.info.ny == r1 - r0 + lo + hi == len(rows)
        assert list(rows[lo:len(rows) - hi]) == list(range(r0, r1))
        y = prob.array("xyz_nodes").reshape(prob.info.n_elem, 2, prob.info.n_s)[:, 1]
        assert abs(y.min() - (r0 - lo) * hy) < 1e-12 and abs(y.max() - (r1 + hi) * hy) < 1e-12


class FakeSlab:
    """A slab whose 'state' rows hold (global row, column) tags in CPU tensors, with the device
    slab's pack / unpack row choices."""

    def __init__(self, dec, i, device=0):
        import torch
        self.index = i
        _, self.lo, self.hi, self.rows = dec.slab(i)
        self.device = torch.device("cpu")
        nyl, nx = len(self.rows), dec.nx
        self.state = np.full((nyl, nx, 3), -1.0)
        own = slice(self.lo, nyl - self.hi)
        self.state[own, :, 0] = self.rows[own][:, None]
        self.state[own, :, 1] = np.arange(nx)[None, :]
        self.state[own, :, 2] = 7.0
        self.send = [torch.zeros(max(g, 1) * nx * 3, dtype=torch.float64) for g in (self.lo, self.hi)]
        self.recv = [torch.zeros(max(g, 1) * nx * 3, dtype=torch.float64) for g in (self.lo, self.hi)]
        self.word = torch.tensor([100 + 37 * i], dtype=torch.int64)

    def pack(self, side):
        nyl = self.state.shape[0]
        r = slice(self.lo, 2 * self.lo) if side == 0 else slice(nyl - 2 * self.hi, nyl - self.hi)
        g = self.lo if side == 0 else self.hi
        self.send[side][:g * self.state[0].size] = __import__("torch").from_numpy(self.state[r].reshape(-1).copy())

    def unpack(self, side, buf):
        nyl = self.state.shape[0]
        g = self.lo if side == 0 else self.hi
        r = slice(0, g) if side == 0 else slice(nyl - g, nyl)
        self.state[r] = buf[:g * self.state[0].size].numpy().reshape(self.state[r].shape)

    def umax(self):
        return self.word

    def stream(self):
        return contextlib.nullcontext()

    def close(self):
        pass

    @property
    def problem(self):
        class _P:
            class info:
                cfl_scaled = 0.01 + 1e-3 * self.index
        return _P

    def set_cfl_scale(self, value):
        self.cfl = value


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, periodic, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        bc = ("periodic", "transmissive", "periodic", "transmissive") if periodic else ("reflective",) * 4
        dec = S.Decomposition(2, 8, 6 * ws, ws, bc=bc, flux="rusanov", limiter="m2l", cfl=0.3)
        run = S.SlabRun(dec, [rank], S.DistTransport(), slab_factory=FakeSlab)
        run.transport.exchange(run)
        run.transport.exchange(run)  # a second round moves the same rows again
        (s,) = run.slabs
        run.transport.reduce_umax(run)
        status = run.transport.reduce_status(run, 3 if rank == ws - 1 else 0)
        assert s.cfl == 0.01 and run.cfl_scaled == 0.01  # the smallest of the slabs' scales
        q.put((rank, s.state.tolist(), s.rows.tolist(), int(s.word.item()), status))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_dist_transport_fills_ghost_rows_gloo(ws, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, periodic, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(ws))
    for rank, state, rows, word, status in got:
        st = np.array(state)
        assert np.all(st[:, :, 0] == np.array(rows)[:, None]), (rank, st[:, 0, 0], rows)  # every row, ghosts too
        assert np.all(st[:, :, 1] == np.arange(8)[None, :]) and np.all(st[:, :, 2] == 7.0)
        assert word == 100 + 37 * (ws - 1)  # the MAX over the slabs
        assert status == 3                   # any slab's failure reaches every rank
