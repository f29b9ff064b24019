"""Slab decomposition of one structured 2D problem over several device contexts.

The grid's rows of elements are split into contiguous y-slabs (the reference splits its mesh over
MPI ranks, simpleMesh.cc:1006-1074).  Each slab is a DGSolver on its own structured grid: the
owned rows plus GHOST rows of elements on every side that has a neighbour slab (both sides when y
is periodic).  Before every stage the ghost rows are refreshed from the neighbours' owned rows --
the reference's ghost exchange before every residual and limiter pass (rk.cc:108-114, 173,
203-209; communicator_cpu.cc:14-59), done per slab boundary instead of per ghost element -- and
the CFL wave speed is max-reduced over the slabs before the step's dt is formed (RK::DtFromCFL over
the whole mesh).  A stage reaches two rows deep (the residual, then the limiter's y pass), so two
ghost rows make every owned row's result the one of the whole grid advanced at once.  (The
sensor-gated limiters are not available here: their flags follow the reference's sequential element
order, a recurrence that can cross any number of rows.)

Transports move the rows:
  LocalTransport  every slab in this process on one device (device-to-device copies)
  DistTransport   one slab per rank over torch.distributed (NCCL for device buffers)
"""
from __future__ import annotations

import contextlib

import numpy as np

from . import _ffi as F
from .solver import DGSolver, Problem

GHOST = 2  # rows of elements: residual (1) + limiter y pass (1)


def tile_rows(order: int) -> int:
    """Height in elements of the tiled 2D residual kernel's tile (32 x 4, or 32 x 2 at p = 3)."""
    return 4 if order <= 2 else 2


def ghost_rows(i: int, nslabs: int, periodic: bool) -> tuple[int, int]:
    """(below, above) ghost rows of slab i."""
    if nslabs == 1:
        return 0, 0
    return (GHOST if periodic or i > 0 else 0), (GHOST if periodic or i < nslabs - 1 else 0)


def neighbours(i: int, nslabs: int, periodic: bool) -> tuple[int | None, int | None]:
    """(slab below, slab above) of slab i, None at a physical boundary."""
    if nslabs == 1:
        return None, None
    lo = i - 1 if i > 0 else (nslabs - 1 if periodic else None)
    hi = i + 1 if i < nslabs - 1 else (0 if periodic else None)
    return lo, hi


def partition_rows(ny: int, nslabs: int, order: int, periodic: bool) -> list[tuple[int, int]]:
    """Owned row ranges [r0, r1) of nslabs near-equal y-slabs of an ny-row grid.  Where possible
    every slab's extent with its ghost rows is a multiple of the residual tile's height, so that
    every slab runs the tiled kernel; each slab owns at least GHOST rows (its neighbours' ghosts)."""
    if nslabs < 1:
        raise ValueError("nslabs >= 1")
    if nslabs > 1 and ny < nslabs * GHOST:
        raise ValueError(f"{ny} rows cannot give {nslabs} slabs of at least {GHOST} rows")
    th = tile_rows(order)
    sizes, done = [], 0
    for i in range(nslabs):
        if i == nslabs - 1:
            sizes.append(ny - done)
            break
        g = sum(ghost_rows(i, nslabs, periodic))
        target = round((i + 1) * ny / nslabs) - done
        rest_min = (nslabs - 1 - i) * GHOST  # rows the later slabs need at least
        cands = [n for n in range(max(GHOST, target - th), target + th + 1)
                 if (n + g) % th == 0 and ny - done - n >= rest_min]
        n = min(cands, key=lambda n: (abs(n - target), n)) if cands else max(GHOST, target)
        sizes.append(n)
        done += n
    if sizes[-1] < (GHOST if nslabs > 1 else 1):
        raise ValueError("no partition with at least GHOST rows per slab")
    out, r = [], 0
    for n in sizes:
        out.append((r, r + n))
        r += n
    return out


class Decomposition:
    """The global structured problem (Problem.structured arguments, 2D) and its y-slabs."""

    def __init__(self, order: int, nx: int, ny: int, nslabs: int, x0=0.0, x1=1.0, y0=0.0, y1=1.0,
                 bc=("transmissive",) * 4, **options):
        bc = tuple(bc)
        if (bc[0] == "periodic") != (bc[2] == "periodic"):
            raise ValueError("bottom and top are both periodic or neither")
        self.order, self.nx, self.ny, self.nslabs = order, nx, ny, nslabs
        self.x0, self.x1, self.y0, self.y1, self.bc = x0, x1, y0, y1, bc
        self.options = options
        self.periodic = bc[0] == "periodic"
        self.ranges = partition_rows(ny, nslabs, order, self.periodic)

    def global_problem(self) -> Problem:
        return Problem.structured(2, self.order, self.nx, self.ny, self.x0, self.x1, self.y0, self.y1, self.bc,
                                  **self.options)

    def slab(self, i: int) -> tuple[Problem, int, int, np.ndarray]:
        """(problem of slab i, ghost rows below, above, global row of each local row)."""
        r0, r1 = self.ranges[i]
        lo, hi = ghost_rows(i, self.nslabs, self.periodic)
        hy = (self.y1 - self.y0) / self.ny
        nyl = r1 - r0 + lo + hi
        bc = (self.bc[0] if lo == 0 else "transmissive", self.bc[1],
              self.bc[2] if hi == 0 else "transmissive", self.bc[3])
        prob = Problem.structured(2, self.order, self.nx, nyl, self.x0, self.x1, self.y0 + (r0 - lo) * hy,
                                  self.y0 + (r1 + hi) * hy, bc, **self.options)
        rows = (np.arange(nyl) + r0 - lo) % self.ny
        return prob, lo, hi, rows


class Slab:
    """One slab on a device: its DGSolver with ghost rows, the rows it covers, its halo buffers."""

    def __init__(self, dec: Decomposition, i: int, device: int = 0):
        import torch
        self.index = i
        self.problem, self.lo, self.hi, self.rows = dec.slab(i)
        self.solver = DGSolver(self.problem, device)
        self.solver.set_ghost_rows(self.lo, self.hi)
        self.device = torch.device("cuda", device)
        self.nx = dec.nx
        info = self.problem.info
        self.per_elem = info.n_fields * info.n_s
        n = [self.solver.halo_count(s) for s in (0, 1)]
        self.send = [torch.empty(max(k, 1), dtype=torch.float64, device=self.device) for k in n]
        self.recv = [torch.empty(max(k, 1), dtype=torch.float64, device=self.device) for k in n]
        self.count = n

    def close(self):
        self.solver.close()

    def set_cfl_scale(self, value: float) -> None:
        self.solver.set_cfl_scale(value)

    # state in the reference layout, rows of elements
    def set_from_global(self, U: np.ndarray) -> None:
        V = np.asarray(U, np.float64).reshape(-1, self.nx, self.per_elem)
        self.solver.set_state(np.ascontiguousarray(V[self.rows]).reshape(-1))

    def owned(self) -> np.ndarray:
        V = self.solver.get_state().reshape(-1, self.nx, self.per_elem)
        return V[self.lo:V.shape[0] - self.hi]

    # halo and reduction hooks used by the transports
    def pack(self, side: int) -> None:
        self.solver.halo_pack(side, self.send[side].data_ptr())

    def unpack(self, side: int, buf) -> None:
        self.solver.halo_unpack(side, buf.data_ptr())

    def umax(self):
        """The step's max-wave-speed word as a 1-element int64 tensor aliasing device memory."""
        import torch
        ptr = self.solver.wavespeed_word()

        class _Word:  # a device array interface over the library's word
            __cuda_array_interface__ = {"shape": (1,), "typestr": "<i8", "data": (ptr, False), "version": 2}
        return torch.as_tensor(_Word(), device=self.device)

    def torch_stream(self):
        """The context's CUDA stream as a torch stream object."""
        import torch
        if getattr(self, "_ts", None) is None:
            self._ts = torch.cuda.ExternalStream(self.solver.stream(), device=self.device)
        return self._ts

    def stream(self):
        import torch
        return torch.cuda.stream(self.torch_stream())

    def record(self):
        """An event recorded on the context's stream now."""
        import torch
        ev = torch.cuda.Event()
        ev.record(self.torch_stream())
        return ev

    def wait(self, ev) -> None:
        """Later work on the context's stream waits for `ev` (no host synchronisation)."""
        self.torch_stream().wait_event(ev)

    def synchronize(self) -> None:
        self.torch_stream().synchronize()


class LocalTransport:
    """Every slab in this process (one device): rows move by device-to-device copies ordered by
    CUDA events between the slabs' streams -- a slab unpacks after its neighbours have packed, and
    packs again only after its neighbours have unpacked -- with no host synchronisation.

    captured=True (default): SlabRun.advance hands the whole sequence to the library
    (dgb_slabs_advance_local), which captures one step of every slab, exchanges included, into one
    CUDA graph and replays it; captured=False drives the phase-level step from here, eagerly."""

    def __init__(self, captured: bool = True):
        self.captured = captured

    def advance(self, run: "SlabRun", nsteps: int, dt: float, scheme: int) -> float:
        """nsteps steps of every slab through the library's captured local step; the time advanced."""
        import ctypes as C
        n = len(run.slabs)
        order = sorted(run.slabs, key=lambda s: s.index)
        handles = (C.c_void_p * n)(*[s.solver._h.value for s in order])
        t = C.c_double(0.0)
        F.check(F.lib().dgb_slabs_advance_local(handles, n, int(run.dec.periodic), int(scheme), int(nsteps),
                                                float(dt), C.byref(t)))
        return t.value

    def exchange(self, run: "SlabRun") -> None:
        packed = {}
        for s in run.slabs:
            for side, g in ((0, s.lo), (1, s.hi)):
                if g:
                    s.pack(side)
            packed[s.index] = s.record()
        by_index = {s.index: s for s in run.slabs}
        unpacked = {}
        for s in run.slabs:
            below, above = neighbours(s.index, run.dec.nslabs, run.dec.periodic)
            for nb in {below, above} - {None}:
                s.wait(packed[nb])
            if below is not None:
                s.unpack(0, by_index[below].send[1])  # the owned top rows of the slab below
            if above is not None:
                s.unpack(1, by_index[above].send[0])
            unpacked[s.index] = s.record()
        for s in run.slabs:  # send buffers are rewritten by the next pack
            below, above = neighbours(s.index, run.dec.nslabs, run.dec.periodic)
            for nb in {below, above} - {None}:
                s.wait(unpacked[nb])

    def reduce_umax(self, run: "SlabRun") -> None:
        """MAX of the slabs' wave-speed words on the device, written back to every word."""
        import torch
        first = run.slabs[0]
        for s in run.slabs[1:]:
            first.wait(s.record())
        with first.stream():
            words = [s.umax() for s in run.slabs]
            m = torch.stack(words).max(dim=0).values
            for w in words:
                w.copy_(m)
        done = first.record()
        for s in run.slabs[1:]:
            s.wait(done)

    def reduce_status(self, run: "SlabRun", code: int) -> int:
        return code

    def reduce_min(self, run: "SlabRun", value: float) -> float:
        return value


class DistTransport:
    """One slab per rank over torch.distributed.  Rows cross in two ordered phases -- every slab
    sends its top rows up and receives its bottom ghosts from below, then the reverse -- so that a
    pair of ranks exchanges one message per direction per phase even when the slab below and the
    slab above are the same rank (two slabs, periodic y).  With NCCL the sends and receives are
    ordered after the slab's own stream and the unpacking after them."""

    def __init__(self, group=None):
        self.group = group
        self._ready = False

    def _p2p(self, ops):
        import torch.distributed as dist
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def _init(self, run):
        import torch
        import torch.distributed as dist
        if not self._ready:  # every rank takes part in the group's first collective
            t = torch.zeros(1, dtype=torch.int64, device=run.slabs[0].device)
            dist.all_reduce(t, group=self.group)
            self._ready = True

    def exchange(self, run: "SlabRun") -> None:
        import torch.distributed as dist
        self._init(run)
        (s,) = run.slabs
        below, above = neighbours(s.index, run.dec.nslabs, run.dec.periodic)
        rank = run.rank_of
        with s.stream():
            if s.hi:
                s.pack(1)
            if s.lo:
                s.pack(0)
            ops = []
            if above is not None:
                ops.append(dist.P2POp(dist.isend, s.send[1], rank(above), group=self.group))
            if below is not None:
                ops.append(dist.P2POp(dist.irecv, s.recv[0], rank(below), group=self.group))
            self._p2p(ops)
            if below is not None:
                s.unpack(0, s.recv[0])
            ops = []
            if below is not None:
                ops.append(dist.P2POp(dist.isend, s.send[0], rank(below), group=self.group))
            if above is not None:
                ops.append(dist.P2POp(dist.irecv, s.recv[1], rank(above), group=self.group))
            self._p2p(ops)
            if above is not None:
                s.unpack(1, s.recv[1])

    def reduce_umax(self, run: "SlabRun") -> None:
        import torch.distributed as dist
        self._init(run)
        (s,) = run.slabs
        with s.stream():
            # reduced in a copy the torch allocator owns (the word itself is the library's memory,
            # which the collective's stream bookkeeping should not be given), then written back
            word = s.umax()
            t = word.clone()
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
            word.copy_(t)

    def reduce_status(self, run: "SlabRun", code: int) -> int:
        import torch
        import torch.distributed as dist
        t = torch.tensor([code], dtype=torch.int64, device=run.slabs[0].device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return int(t.item())

    def reduce_min(self, run: "SlabRun", value: float) -> float:
        import torch
        import torch.distributed as dist
        t = torch.tensor([value], dtype=torch.float64, device=run.slabs[0].device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class SlabRun:
    """The slabs of a decomposition that live in this process, advanced together.

    local:  SlabRun(dec, range(dec.nslabs), LocalTransport())            one process, one GPU
    ranks:  SlabRun(dec, [rank], DistTransport(), device=local_rank)       one slab per rank
    """

    def __init__(self, dec: Decomposition, slabs, transport, device: int = 0, slab_factory=Slab):
        self.dec = dec
        self.transport = transport
        self.slabs = [slab_factory(dec, i, device) for i in slabs]
        self.rank_of = lambda i: i  # slab i lives on rank i
        # one CFL scale for every slab: the smallest of the slabs' own (their meshes can give it
        # one ulp apart), as the whole grid's smallest element sets it
        scale = transport.reduce_min(self, min(s.problem.info.cfl_scaled for s in self.slabs))
        for s in self.slabs:
            s.set_cfl_scale(scale)
        self.cfl_scaled = scale

    def close(self):
        for s in self.slabs:
            s.close()

    def set_global_state(self, U: np.ndarray) -> None:
        for s in self.slabs:
            s.set_from_global(U)

    def global_state(self) -> np.ndarray:
        """The whole grid's state (reference layout) from the slabs of this process; all of them
        must be here."""
        if len(self.slabs) != self.dec.nslabs:
            raise ValueError("global_state needs every slab in this process")
        return np.concatenate([s.owned() for s in sorted(self.slabs, key=lambda s: s.index)]).reshape(-1)

    def advance(self, nsteps: int, dt: float = 0.0, scheme: int = F.SSPRK3) -> float:
        """nsteps steps of the whole grid (dt <= 0: the CFL step of the whole grid); returns the
        time advanced.  Raises DGBError on every rank when any slab's step failed."""
        if getattr(self.transport, "captured", False) and len(self.slabs) == self.dec.nslabs:
            return self.transport.advance(self, nsteps, dt, scheme)
        nst = 4 if scheme == F.RK4 else 3
        t = 0.0
        for _ in range(nsteps):
            for s in self.slabs:
                s.solver.step_begin(scheme, dt)
            if not dt > 0:
                self.transport.reduce_umax(self)
            for k in range(nst):
                self.transport.exchange(self)
                for s in self.slabs:
                    s.solver.step_stage(k)
            codes = [s.solver.step_end() for s in self.slabs]
            rc = self.transport.reduce_status(self, max(c for c, _ in codes))
            if rc:
                raise F.DGBError(rc, F.lib().dgb_last_error().decode() or "a slab's step failed")
            t += codes[0][1]
        return t

    @contextlib.contextmanager
    def closing(self):
        try:
            yield self
        finally:
            self.close()
