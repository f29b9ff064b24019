"""Host-side mirror of the reference's solver objects over the C ABI.

The reference drives its hot path through C++ objects built in code/src/main.cc:
``DG_SOLVER`` (code/src/dg/dg_solver.h:104, ``dg_solver()`` at :292), ``Limiting``
(code/src/limiting/limiting.h:123/249), ``RK`` (code/src/time_integration/rk.h:27,
``RK_integration`` rk.cc:11, ``DtFromCFL`` rk.cc:250).  ``Problem`` and ``DGSolver`` below expose
the same operations on the B200 path with the same argument meaning; states are float64 arrays in
the reference layout ``U[(e*N_F+f)*N_s+i]`` (main.cc:814-820).  Failures the reference turns into
``exit(1)`` raise :class:`DGBError` with the C status code.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

from . import _ffi as F


class Problem:
    """Deck + mesh + basis/quadrature/geometry setup (main.cc:273-860), host only."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._destroy = F.lib().dgb_problem_destroy  # bound now: module globals are gone at interpreter exit
        info = F.Info()
        F.check(F.lib().dgb_problem_info(self._h, C.byref(info)))
        self.info = info

    @classmethod
    def from_deck(cls, deck: str | Path) -> "Problem":
        h = C.c_void_p()
        F.check(F.lib().dgb_problem_from_deck(str(deck).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def structured(cls, dim: int, order: int, nx: int, ny: int = 1, x0: float = 0.0, x1: float = 1.0,
                   y0: float = 0.0, y1: float = 1.0, bc: Sequence[str | int] = ("transmissive",) * 4,
                   flux: str = "roe", limiter: str = "m2l", cfl: float = -1.0,
                   thresholds: Iterable[float] = (), n_mass: int = 0, gamma_model: str = "gamncon") -> "Problem":
        spec = mesh_spec(dim, order, nx, ny, x0, x1, y0, y1, bc)
        opt = F.Options()
        opt.n_mass = int(n_mass)
        opt.gamma_model = F.GAMMA_MODEL[gamma_model.lower()]
        opt.flux = F.FLUX[flux.lower()]
        opt.limiter = F.LIMITER[limiter.lower()]
        opt.cfl = cfl
        th = list(thresholds)[:3]
        for k, t in enumerate(th):
            opt.thresholds[k] = t
        opt.n_thresholds = len(th)
        h = C.c_void_p()
        F.check(F.lib().dgb_problem_structured(C.byref(spec), C.byref(opt), C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = None

    @property
    def state_size(self) -> int:
        i = self.info
        return i.n_elem * i.n_fields * i.n_s

    def array(self, name: str) -> np.ndarray:
        n = C.c_size_t()
        F.check(F.lib().dgb_problem_array_size(self._h, name.encode(), C.byref(n)))
        ints = name in ("map", "invmap", "boundaryMap", "neighbors", "tensor_perm")
        a = np.zeros(n.value // (4 if ints else 8), np.int32 if ints else np.float64)
        F.check(F.lib().dgb_problem_get_array(self._h, name.encode(), a.ctypes.data_as(C.c_void_p), n.value))
        return a

    def init_state(self, ic: str, params: Sequence[float] = (), seed: int = 0) -> np.ndarray:
        U = np.zeros(self.state_size)
        prm = np.asarray(list(params), np.float64)
        F.check(F.lib().dgb_problem_init_state(self._h, ic.encode(), F.dptr(prm) if prm.size else None,
                                               int(prm.size), int(seed), F.dptr(U)))
        return U

    def error_norms(self, U, U_exact) -> dict:
        """The reference driver's ERROR diagnostic (main.cc:909-1038): dx and the L1, L2, Linf per
        field of the cell averages of U against U_exact."""
        U = np.ascontiguousarray(U, np.float64)
        Ue = np.ascontiguousarray(U_exact, np.float64)
        nf = self.info.n_fields
        out = np.zeros(1 + 3 * nf)
        F.check(F.lib().dgb_problem_error_norms(self._h, F.dptr(U), F.dptr(Ue), F.dptr(out)))
        return {"dx": out[0], "l1": out[1:1 + nf], "l2": out[1 + nf:1 + 2 * nf], "linf": out[1 + 2 * nf:]}

    def write_pos(self, U: np.ndarray, step: int, time: float, directory: str | Path) -> None:
        U = np.ascontiguousarray(U, np.float64)
        F.check(F.lib().dgb_write_pos(self._h, F.dptr(U), int(step), float(time), str(directory).encode()))

    def read_pos(self, step: int, directory: str | Path) -> tuple[np.ndarray, float]:
        U = np.zeros(self.state_size)
        t = C.c_double()
        F.check(F.lib().dgb_read_pos(self._h, int(step), str(directory).encode(), C.byref(t), F.dptr(U)))
        return U, t.value


def mesh_spec(dim, order, nx, ny=1, x0=0.0, x1=1.0, y0=0.0, y1=1.0, bc=("transmissive",) * 4) -> F.MeshSpec:
    s = F.MeshSpec()
    s.dim, s.order, s.nx, s.ny = dim, order, nx, ny
    s.x0, s.x1, s.y0, s.y1 = x0, x1, y0, y1
    for k, b in enumerate(list(bc)[:4]):
        s.bc[k] = b if isinstance(b, int) else F.BC[b]
    return s


def write_msh(path: str | Path, dim, order, nx, ny=1, x0=0.0, x1=1.0, y0=0.0, y1=1.0,
              bc=("transmissive",) * 4) -> None:
    """Gmsh 2.2 file of a structured mesh (element order row-major, boundary tags bc)."""
    spec = mesh_spec(dim, order, nx, ny, x0, x1, y0, y1, bc)
    F.check(F.lib().dgb_mesh_write_msh(C.byref(spec), str(path).encode()))


class DGSolver:
    """Device context: DG_SOLVER + Limiting + RK of the reference, on one GPU."""

    def __init__(self, problem: Problem, device: int = 0):
        self.problem = problem
        self._destroy = F.lib().dgb_destroy
        self._h = C.c_void_p()
        F.check(F.lib().dgb_create(problem._h, int(device), C.byref(self._h)))
        self.n = problem.state_size

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _arr(self, U) -> np.ndarray:
        U = np.ascontiguousarray(U, np.float64)
        if U.size != self.n:
            raise ValueError(f"state has {U.size} values, expected {self.n}")
        return U

    def set_state(self, U) -> None:
        F.check(F.lib().dgb_set_state(self._h, F.dptr(self._arr(U))))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """The resident state (reference layout).  `out`: a contiguous float64 array of the state's
        size to read into (pinned host memory makes the device-to-host copy a direct DMA)."""
        if out is None:
            U = np.empty(self.n)
        else:
            U = out
            if U.dtype != np.float64 or U.size != self.n or not U.flags.c_contiguous:
                raise ValueError(f"out must be a contiguous float64 array of {self.n} values")
        F.check(F.lib().dgb_get_state(self._h, F.dptr(U)))
        return U

    def dg_solver(self, U) -> np.ndarray:
        """f = S + F + Q (DG_SOLVER::dg_solver)."""
        f = np.zeros(self.n)
        F.check(F.lib().dgb_residual(self._h, F.dptr(self._arr(U)), F.dptr(f)))
        return f

    def solve(self, dt: float, U) -> np.ndarray:
        """DU = dt Minv f(U) (Lsolver applied to dg_solver's output)."""
        DU = np.zeros(self.n)
        F.check(F.lib().dgb_solve(self._h, float(dt), F.dptr(self._arr(U)), F.dptr(DU)))
        return DU

    def limit(self, U) -> np.ndarray:
        """Limited copy of U with the problem's limiter (Limiting::*limiting)."""
        V = self._arr(U).copy()
        F.check(F.lib().dgb_limit(self._h, F.dptr(V)))
        return V

    def set_form(self, form: str) -> None:
        """Arithmetic of the residual: "fp64" (plain, the parity form) or "mixed" (FP32 contractions
        and fluxes on FP64 anchors, FP64 pressure recovery and stage update)."""
        F.check(F.lib().dgb_set_form(self._h, F.FORM[form]))

    def set_wait_limit(self, polls: int = 1 << 22) -> None:
        """Poll budget of the residual kernels' first wait on each tile copy (0: give up at once,
        which makes the next step fail with DGB_ERR_TIMEOUT; the default restores the normal
        budget)."""
        F.check(F.lib().dgb_set_wait_limit(self._h, int(polls)))

    def sensors(self, U) -> np.ndarray:
        """Troubled-cell flags of U (SENSOR::sensing): 0 or the number of the sensor that fired."""
        flags = np.zeros(self.problem.info.n_elem, np.int32)
        F.check(F.lib().dgb_sensors(self._h, F.dptr(self._arr(U)), flags.ctypes.data_as(C.POINTER(C.c_int))))
        return flags

    def dt_from_cfl(self, U) -> float:
        dt = C.c_double()
        F.check(F.lib().dgb_dt_from_cfl(self._h, F.dptr(self._arr(U)), C.byref(dt)))
        return dt.value

    def advance(self, nsteps: int, dt: float = 0.0, scheme: int = F.SSPRK3) -> float:
        """Advances the resident state; returns the time advanced (RK::RK_integration loop)."""
        t = C.c_double(0.0)
        F.check(F.lib().dgb_advance(self._h, int(scheme), int(nsteps), float(dt), C.byref(t)))
        return t.value

    def advance_host(self, U: np.ndarray, nsteps: int, dt: float = 0.0, scheme: int = F.SSPRK3) -> float:
        """Advances nsteps steps with the state of record in the host array U (reference layout,
        contiguous float64, updated in place): every step uploads U, advances one step and
        downloads the result into U (dgb_advance_host).  Returns the time advanced."""
        if U.dtype != np.float64 or U.size != self.n or not U.flags.c_contiguous or not U.flags.writeable:
            raise ValueError(f"U must be a writable contiguous float64 array of {self.n} values")
        t = C.c_double(0.0)
        F.check(F.lib().dgb_advance_host(self._h, F.dptr(U), int(scheme), int(nsteps), float(dt), C.byref(t)))
        return t.value

    def last_timing(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_longlong()
        F.check(F.lib().dgb_last_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_profiling(self, on: bool) -> None:
        F.check(F.lib().dgb_set_profiling(self._h, 1 if on else 0))

    def kernel_timing(self, name: str) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_longlong()
        F.check(F.lib().dgb_kernel_timing(self._h, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def conservation(self) -> np.ndarray:
        tot = np.zeros(self.problem.info.n_fields)
        F.check(F.lib().dgb_conservation(self._h, F.dptr(tot)))
        return tot

    # --- slab mode and the phase-level step (dgb_slab_ghost_rows, dgb_step_*, dgb_halo_*) ---------
    def set_ghost_rows(self, lo: int, hi: int) -> None:
        F.check(F.lib().dgb_slab_ghost_rows(self._h, int(lo), int(hi)))

    def set_cfl_scale(self, cfl_scaled: float) -> None:
        F.check(F.lib().dgb_set_cfl_scale(self._h, float(cfl_scaled)))

    def step_begin(self, scheme: int, dt: float) -> None:
        F.check(F.lib().dgb_step_begin(self._h, int(scheme), float(dt)))

    def wavespeed_word(self) -> int:
        """Device address of the step's max-wave-speed word (uint64 bits of a non-negative double)."""
        p = C.c_void_p()
        F.check(F.lib().dgb_step_wavespeed_word(self._h, C.byref(p)))
        return int(p.value)

    def step_stage(self, k: int) -> None:
        F.check(F.lib().dgb_step_stage(self._h, int(k)))

    def step_end(self) -> tuple[int, float]:
        """(status, dt of the step); the status is not raised so that slabs can agree on it first."""
        t = C.c_double(0.0)
        rc = F.lib().dgb_step_end(self._h, C.byref(t))
        return rc, t.value

    def halo_count(self, side: int) -> int:
        n = C.c_size_t()
        F.check(F.lib().dgb_halo_count(self._h, int(side), C.byref(n)))
        return n.value

    def halo_pack(self, side: int, dst_ptr: int) -> None:
        F.check(F.lib().dgb_halo_pack(self._h, int(side), C.c_void_p(dst_ptr)))

    def halo_unpack(self, side: int, src_ptr: int) -> None:
        F.check(F.lib().dgb_halo_unpack(self._h, int(side), C.c_void_p(src_ptr)))

    def stream(self) -> int:
        """The context's cudaStream_t as an integer."""
        p = C.c_void_p()
        F.check(F.lib().dgb_stream(self._h, C.byref(p)))
        return int(p.value or 0)


class DGBatch:
    """Batched ensemble (dgb_batch_*): independent problems, one DGSolver each, advanced together
    with SSP-RK3, every case with its own CFL step.  The solvers stay usable on their own (states
    are set and read through them) and must outlive the batch."""

    CLASS_KEYS = ("dim", "order", "flux", "limiter", "cases", "tile_w", "tile_h", "unroll", "ctas_per_sm",
                  "tuned_ns")

    def __init__(self, solvers: Sequence["DGSolver"]):
        self.solvers = list(solvers)
        self._destroy = F.lib().dgb_batch_destroy
        arr = (C.c_void_p * len(self.solvers))(*[s._h for s in self.solvers])
        self._h = C.c_void_p()
        F.check(F.lib().dgb_batch_create(arr, len(self.solvers), C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def classes(self) -> list[dict]:
        out = []
        for k in range(F.lib().dgb_batch_n_classes(self._h)):
            info = (C.c_int * 10)()
            F.check(F.lib().dgb_batch_class_info(self._h, k, info))
            out.append(dict(zip(self.CLASS_KEYS, list(info))))
        return out

    def autotune(self, reps: int = 5) -> list[dict]:
        F.check(F.lib().dgb_batch_autotune(self._h, int(reps)))
        return self.classes()

    def set_tuning(self, k: int, tile_w: int, tile_h: int = 1, unroll: int = 1, ctas_per_sm: int = 0) -> None:
        F.check(F.lib().dgb_batch_set_tuning(self._h, int(k), int(tile_w), int(tile_h), int(unroll), int(ctas_per_sm)))

    def advance(self, nsteps: int, t_end: float = 0.0) -> int:
        n = C.c_int()
        F.check(F.lib().dgb_batch_advance(self._h, int(nsteps), float(t_end), C.byref(n)))
        return n.value

    def case_stats(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(simulated time, steps, wall ms to the stop at t_end or -1) per case of the last run."""
        n = len(self.solvers)
        t, w = np.zeros(n), np.zeros(n)
        s = np.zeros(n, np.int32)
        F.check(F.lib().dgb_batch_case_stats(self._h, F.dptr(t), s.ctypes.data_as(C.POINTER(C.c_int)), F.dptr(w)))
        return t, s, w

    def last_timing(self) -> tuple[float, int]:
        ms, n = C.c_double(), C.c_longlong()
        F.check(F.lib().dgb_batch_last_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value
