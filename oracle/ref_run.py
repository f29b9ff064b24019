"""Driver for the reference CPU oracle binaries built by oracle/build_ref.py (test infrastructure).

Writes a Gmsh mesh and a reference input deck into a work directory, runs
``oracle/_ref/dgref_<dim>d_<flux> -d deck.inp --cmd <cmd>`` (see oracle/ref_harness.cc) on a
state file and reads the result back.  Only tests, fixture generation and the CPU-baseline leg
of bench.py use this module.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

FLUX_TAG = {"rusanov": "rus", "rus": "rus", "roe": "roe", "hll": "hll"}
BC_TAG = {"periodic": 1, "transmissive": 2, "reflective": 3, "frozen": 4}


def binary(dim: int, flux: str, n_mass: int = 0, error: bool = False, gamcons: bool = False,
           cons: bool = False) -> Path:
    """The reference build for (dimension, flux) with N_Y = n_mass (0 or 1) mass fractions, with
    the ERROR or CONS diagnostic compiled in, or with the GAMCONS gamma model."""
    return REF_DIR / (f"dgref_{dim}d_{FLUX_TAG[flux.lower()]}" + (f"_y{n_mass}" if n_mass else "") +
                      ("_err" if error else "") + ("_gc" if gamcons else "") + ("_cons" if cons else ""))


def available(dim: int = 2, flux: str = "rusanov", n_mass: int = 0, gamcons: bool = False) -> bool:
    return binary(dim, flux, n_mass, gamcons=gamcons).exists()


@dataclass
class RefCase:
    dim: int
    order: int
    nx: int
    ny: int = 1
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    bc: tuple = ("transmissive",) * 4
    flux: str = "rusanov"
    limiter: str = "m2l"
    cfl: float = -1.0
    output_times: tuple = (0.0, 1e-3)
    thresholds: tuple = ()
    n_mass: int = 0
    ic: str = ""                  # deck "#initial condition" (default sodtube / sodcirc)
    make_options: tuple = ()      # "#Make options" KEY=VALUE lines (read by dgbexec, ignored by the reference)
    error: bool = False           # run the build with the ERROR diagnostic
    gamcons: bool = False         # run the GAMCONS build
    cons: bool = False            # run the build with the CONS diagnostic
    workdir: Path | None = None
    _tmp: object = field(default=None, repr=False)

    def __post_init__(self):
        if self.workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="dgref_")
            self.workdir = Path(self._tmp.name)
        self.workdir = Path(self.workdir)
        self.workdir.mkdir(parents=True, exist_ok=True)
        from oracle.workload import structured_msh  # the mesh file is an input to both codes
        structured_msh(self.workdir / "mesh.msh", self.dim, self.order, self.nx, self.ny, self.x0, self.x1,
                       self.y0, self.y1, self.bc)
        self.write_deck()

    def write_deck(self, cfl: float | None = None, output_times=None) -> Path:
        cfl = self.cfl if cfl is None else cfl
        out = self.output_times if output_times is None else output_times
        lines = (["#Make options", *self.make_options] if self.make_options else []) + [
                 "#Code options", "#time integration", "rk4", "#output time array",
                 " ".join(repr(float(t)) for t in out), "#final time", repr(float(out[-1])),
                 "#Courant-Friedrichs-Lewy condition", repr(float(cfl)), "#order", str(self.order),
                 "#mesh file", "mesh.msh", "lin" if self.dim == 1 else "qua", "#limiter", self.limiter,
                 "#initial condition", self.ic or ("sodtube" if self.dim == 1 else "sodcirc")]
        if self.thresholds:
            lines += ["#sensor thresholds", " ".join(repr(float(t)) for t in self.thresholds)]
        p = self.workdir / "deck.inp"
        p.write_text("\n".join(lines) + "\n")
        return p

    def run(self, cmd: str, U: np.ndarray | None = None, dt: float = 0.0, nsteps: int = 1,
            repeat: int = 1, timeout: float = 600.0, extra_env: dict | None = None) -> tuple[np.ndarray, str]:
        exe = binary(self.dim, self.flux, self.n_mass, self.error, self.gamcons, self.cons)
        if not exe.exists():
            raise FileNotFoundError(f"{exe} missing: run python oracle/build_ref.py")
        args = [str(exe), "-d", "deck.inp", "--cmd", cmd, "--dt", repr(float(dt)), "--nsteps", str(nsteps),
                "--repeat", str(repeat)]
        if U is not None:
            np.ascontiguousarray(U, np.float64).tofile(self.workdir / "in.bin")
            args += ["--in", "in.bin"]
        args += ["--out", "out.bin", "--dir", "."]
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        if extra_env:
            env.update(extra_env)
        r = subprocess.run(args, cwd=self.workdir, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{' '.join(args)} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        out = self.workdir / "out.bin"
        res = np.fromfile(out) if out.exists() else np.zeros(0)
        return res, r.stdout

    def dump(self) -> dict:
        self.run("dump")
        d = {}
        for f in self.workdir.glob("*.bin"):
            if f.stem in ("in", "out"):
                continue
            ints = f.stem in ("map", "invmap", "neighbors", "boundaryMap")
            d[f.stem] = np.fromfile(f, np.int32 if ints else np.float64)
        meta = {}
        for line in (self.workdir / "meta.txt").read_text().splitlines():
            k, v = line.split()
            meta[k] = float(v) if "." in v or "e" in v else int(v)
        d["meta"] = meta
        return d

    def residual(self, U):
        return self.run("residual", U)[0]

    def solve(self, U, dt):
        return self.run("solve", U, dt=dt)[0]

    def limit(self, U):
        return self.run("limit", U)[0]

    def sensors(self, U):
        return self.run("sensors", U)[0].astype(np.int64)

    def dt_cfl(self, U, cfl):
        self.write_deck(cfl=cfl)
        try:
            return float(self.run("dt", U)[0][0])
        finally:
            self.write_deck()

    def rk4(self, U, dt, nsteps, cfl: float | None = None):
        """nsteps reference RK4 steps; dt <= 0 takes the CFL step from a deck with CFL `cfl`."""
        if cfl is not None:
            self.write_deck(cfl=cfl)
        try:
            return self.run("rk4n", U, dt=dt, nsteps=nsteps)[0]
        finally:
            self.write_deck()

    def rk3(self, U, dt, nsteps, cfl: float | None = None):
        if cfl is not None:
            self.write_deck(cfl=cfl)
        try:
            return self.run("rk3", U, dt=dt, nsteps=nsteps)[0]
        finally:
            self.write_deck()

    def rk4_loop(self, U, dt, nsteps) -> tuple[np.ndarray, float]:
        """The reference time loop itself (RK::RK_integration) over output times k*dt; returns the
        state and the loop's wall time (s)."""
        times = [k * dt for k in range(nsteps + 1)]
        self.write_deck(cfl=-1.0, output_times=times)
        try:
            out, log = self.run("rk4", U)
        finally:
            self.write_deck()
        wall = float(log.split("DGREF_WALL_S")[1].split()[0])
        return out, wall
