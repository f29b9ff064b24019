"""Generates the golden fixtures in tests/golden/*.npz from the reference CPU build.

Each case is a small structured mesh (written with the package's Gmsh writer, read by the
reference's own reader) and a seeded state Uraw; U0 is Uraw after the reference limiter (or Uraw
when the case has no limiter).  The reference binaries of oracle/build_ref.py
(compiled from the reference sources) compute, on that state:
    f      DG_SOLVER::dg_solver                 (code/src/dg/dg_solver.h:292)
    DU     dt * Minv * f                        (Lsolver, code/src/time_integration/rk_kernels.cu:182)
    Ulim   the deck's limiter on the raw state Uraw (Limiting::M2limiting / HRlimiting, limiting.cc)
    dt     RK::DtFromCFL at CFL `cfl`           (code/src/time_integration/rk.cc:250)
    rk4    `nsteps` reference RK4 steps, step `dt_fixed`      (rk.cc:155-209)
    rk3    `nsteps` SSP-RK3 steps of reference operators, step `dt_fixed`
    rk3c   `nsteps` SSP-RK3 steps with the CFL step
plus the reference's setup arrays (phi, ..., Minv, neighbours) for the host-setup pins.

Run from the repository root after `python oracle/build_ref.py` and `python -m dg_b200.build`:
    python tests/golden/make_golden.py [name ...]     (no names: every fixture)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.ref_run import RefCase  # noqa: E402
import dg_b200 as dgb  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = [
    # name, dim, order, nx, ny, domain, bc, flux, limiter, ic, cfl, dt_fixed, nsteps
    dict(name="d1_p2_roe_m2l", dim=1, order=2, nx=24, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="m2l", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5),
    dict(name="d1_p1_rus_hrl_wall", dim=1, order=1, nx=20, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="rusanov", limiter="hrl", ic="tube_noise", cfl=0.4, dt=5e-4, nsteps=5),
    dict(name="d1_p3_hll_m2l_periodic", dim=1, order=3, nx=16, ny=1, dom=(0, 1, 0, 1), bc=("periodic",) * 2,
         flux="hll", limiter="m2l", ic="tube_noise", cfl=0.3, dt=2e-4, nsteps=5),
    dict(name="d1_p2_rus_none", dim=1, order=2, nx=18, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="rusanov", limiter="none", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5),
    dict(name="d2_p2_rus_m2l", dim=2, order=2, nx=8, ny=4, dom=(0, 2, 0, 1), bc=("transmissive",) * 4,
         flux="rusanov", limiter="m2l", ic="shock_bubble", cfl=0.3, dt=1e-3, nsteps=4),
    dict(name="d2_p2_roe_m2l_walls", dim=2, order=2, nx=8, ny=4, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"),
         flux="roe", limiter="m2l", ic="shock_bubble", cfl=0.3, dt=1e-3, nsteps=4),
    dict(name="d2_p1_rus_hrl_periodic", dim=2, order=1, nx=6, ny=6, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="rusanov", limiter="hrl", ic="quadrants", cfl=0.3, dt=1e-3, nsteps=4),
    dict(name="d2_p3_roe_m2l", dim=2, order=3, nx=6, ny=4, dom=(0, 2, 0, 1), bc=("transmissive",) * 4,
         flux="roe", limiter="m2l", ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4),
    dict(name="d2_p2_rus_hrl_box", dim=2, order=2, nx=6, ny=6, dom=(0, 1, 0, 1), bc=("reflective",) * 4,
         flux="rusanov", limiter="hrl", ic="quadrants", cfl=0.3, dt=1e-3, nsteps=4),
    dict(name="d2_p2_roe_none", dim=2, order=2, nx=5, ny=3, dom=(0, 2, 0, 1), bc=("transmissive",) * 4,
         flux="roe", limiter="none", ic="quadrants", cfl=0.3, dt=1e-3, nsteps=3),
    # grids whose extents are multiples of the 32 x 4 element tile (tiled residual kernel)
    dict(name="t2_p2_rus_m2l_walls", dim=2, order=2, nx=32, ny=8, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"),
         flux="rusanov", limiter="m2l", ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4),
    dict(name="t2_p1_roe_hrl_periodic", dim=2, order=1, nx=64, ny=8, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="hrl", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=4),
    dict(name="t2_p2_roe_m2l_box", dim=2, order=2, nx=32, ny=12, dom=(0, 1, 0, 1), bc=("reflective",) * 4,
         flux="roe", limiter="m2l", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=4),
    # sensor-gated limiters (per-element HR / m2 / primitive HR / p=0 on flagged elements) and the
    # primitive-variable HR limiter; thresholds are the deck's "#sensor thresholds"
    dict(name="s2_p2_rus_hri_walls", dim=2, order=2, nx=12, ny=8, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"), flux="rusanov", limiter="hri",
         ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=3, thresholds=(0.01, 0.05, 0.01)),
    dict(name="s2_p2_roe_m2i_periodic", dim=2, order=2, nx=12, ny=8, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="m2i", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=3, thresholds=(0.02, 0.02, 0.02)),
    dict(name="s2_p2_rus_m2i_box", dim=2, order=2, nx=10, ny=10, dom=(0, 1, 0, 1), bc=("reflective",) * 4,
         flux="rusanov", limiter="m2i", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=3, thresholds=(0.02, 0.05)),
    dict(name="s2_p1_roe_pri", dim=2, order=1, nx=10, ny=6, dom=(0, 1, 0, 1), bc=("transmissive",) * 4,
         flux="roe", limiter="pri", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=3, thresholds=(0.02, 0.02)),
    dict(name="s2_p2_rus_p0i", dim=2, order=2, nx=12, ny=8, dom=(0, 2, 0, 1), bc=("transmissive",) * 4,
         flux="rusanov", limiter="p0i", ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=3, thresholds=(0.05,)),
    dict(name="s1_p2_roe_m2i", dim=1, order=2, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="m2i", ic="tube_noise", cfl=0.3, dt=2e-4, nsteps=4, thresholds=(0.01, 0.01, 0.01)),
    dict(name="s1_p3_hll_hri_wall", dim=1, order=3, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="hll", limiter="hri", ic="tube_noise", cfl=0.15, dt=1e-4, nsteps=4, thresholds=(0.01, 0.05)),
    dict(name="s1_p2_rus_pri_periodic", dim=1, order=2, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("periodic",) * 2,
         flux="rusanov", limiter="pri", ic="tube_noise", cfl=0.3, dt=2e-4, nsteps=4, thresholds=(0.001,)),
    dict(name="s1_p2_rus_prl", dim=1, order=2, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="rusanov", limiter="prl", ic="tube_noise", cfl=0.3, dt=2e-4, nsteps=4),
    # one passive mass fraction (the reference built with MASS=1: N_Y = 1)
    dict(name="y1_p2_roe_m2l", dim=1, order=2, nx=24, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="m2l", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5, n_mass=1),
    dict(name="y1_p3_hll_hrl_wall", dim=1, order=3, nx=20, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="hll", limiter="hrl", ic="tube_noise", cfl=0.2, dt=2e-4, nsteps=5, n_mass=1),
    dict(name="y1_p1_rus_m2l_periodic", dim=1, order=1, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("periodic",) * 2,
         flux="rusanov", limiter="m2l", ic="riemann", cfl=0.4, dt=4e-4, nsteps=5, n_mass=1),
    dict(name="y2_p2_rus_m2l_walls", dim=2, order=2, nx=32, ny=8, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"), flux="rusanov", limiter="m2l",
         ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4, n_mass=1),
    dict(name="y2_p2_roe_hrl_periodic", dim=2, order=2, nx=32, ny=8, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="hrl", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=4, n_mass=1),
    dict(name="y2_p1_roe_m2l_box", dim=2, order=1, nx=32, ny=4, dom=(0, 1, 0, 1), bc=("reflective",) * 4,
         flux="roe", limiter="m2l", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=4, n_mass=1),
    # two and three mass fractions (MASS=2, MASS=3; Y_k marks the region for even k, its complement
    # for odd k)
    dict(name="m2_d1_p2_roe_m2l", dim=1, order=2, nx=24, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="m2l", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5, n_mass=2),
    dict(name="m3_d1_p3_hll_hrl_wall", dim=1, order=3, nx=20, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="hll", limiter="hrl", ic="riemann", cfl=0.2, dt=2e-4, nsteps=5, n_mass=3),
    dict(name="m2_d2_p2_rus_m2l_walls", dim=2, order=2, nx=32, ny=8, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"), flux="rusanov", limiter="m2l",
         ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4, n_mass=2),
    dict(name="m3_d2_p1_roe_hrl_periodic", dim=2, order=1, nx=32, ny=4, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="hrl", ic="quadrants", cfl=0.3, dt=5e-4, nsteps=4, n_mass=3),
    # the conservative gamma model (the reference built with GAMM=GAMCONS); its M2limiting stops
    # the run for this model, so the limiters are hrl and none
    dict(name="g1_p2_roe_hrl", dim=1, order=2, nx=24, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="hrl", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5, gamma_model="gamcons"),
    dict(name="g1_p3_hll_none_wall", dim=1, order=3, nx=20, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="hll", limiter="none", ic="tube_noise", cfl=0.05, dt=2e-4, nsteps=5, gamma_model="gamcons"),
    dict(name="g1_p1_rus_hrl_periodic", dim=1, order=1, nx=30, ny=1, dom=(0, 1, 0, 1), bc=("periodic",) * 2,
         flux="rusanov", limiter="hrl", ic="riemann", cfl=0.4, dt=4e-4, nsteps=5, gamma_model="gamcons"),
    dict(name="g2_p2_rus_hrl_walls", dim=2, order=2, nx=32, ny=8, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"), flux="rusanov", limiter="hrl",
         ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4, gamma_model="gamcons"),
    dict(name="g2_p1_roe_none_periodic", dim=2, order=1, nx=32, ny=4, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="none", ic="quadrants", cfl=0.1, dt=5e-4, nsteps=4, gamma_model="gamcons"),
    dict(name="g2_p3_roe_hrl", dim=2, order=3, nx=32, ny=4, dom=(0, 2, 0, 1), bc=("transmissive",) * 4,
         flux="roe", limiter="hrl", ic="shock_bubble", cfl=0.3, dt=2.5e-4, nsteps=4, gamma_model="gamcons"),
    # five and ten mass fractions in 1D (MASS=5, MASS=10)
    dict(name="m10_d1_p2_roe_m2l", dim=1, order=2, nx=24, ny=1, dom=(0, 1, 0, 1), bc=("transmissive",) * 2,
         flux="roe", limiter="m2l", ic="tube_noise", cfl=0.4, dt=4e-4, nsteps=5, n_mass=10),
    dict(name="m5_d1_p3_rus_hrl_wall", dim=1, order=3, nx=20, ny=1, dom=(0, 1, 0, 1), bc=("reflective",) * 2,
         flux="rusanov", limiter="hrl", ic="riemann", cfl=0.2, dt=2e-4, nsteps=5, n_mass=5),
    # ten and five in 2D (tile-aligned: the device path takes mass fractions on full tiles)
    dict(name="m10_d2_p2_rus_m2l_walls", dim=2, order=2, nx=32, ny=4, dom=(0, 2, 0, 1),
         bc=("reflective", "transmissive", "reflective", "transmissive"), flux="rusanov", limiter="m2l",
         ic="shock_bubble", cfl=0.3, dt=5e-4, nsteps=4, n_mass=10),
    dict(name="m5_d2_p3_roe_hrl_periodic", dim=2, order=3, nx=32, ny=4, dom=(0, 1, 0, 1), bc=("periodic",) * 4,
         flux="roe", limiter="hrl", ic="quadrants", cfl=0.3, dt=2.5e-4, nsteps=4, n_mass=5),
]


def perturbed_state(prob: "dgb.Problem", ic: str, seed: int) -> np.ndarray:
    """Seeded IC plus a 1% nodal perturbation of density, momentum and energy (positivity kept)."""
    U = prob.init_state(ic, seed=seed)
    i = prob.info
    V = U.reshape(i.n_elem, i.n_fields, i.n_s)
    rng = np.random.default_rng(seed + 1000)
    nmom = i.dim
    rho = V[:, 0, :] * (1 + 0.01 * rng.uniform(-1, 1, V[:, 0, :].shape))
    V[:, 1:1 + nmom, :] += 0.01 * rng.uniform(-1, 1, V[:, 1:1 + nmom, :].shape) * rho[:, None, :]
    V[:, 0, :] = rho
    V[:, 1 + nmom, :] *= 1 + 0.01 * rng.uniform(-1, 1, V[:, 1 + nmom, :].shape)
    return V.reshape(-1).copy()


def make_case(c: dict, seed: int) -> dict:
    x0, x1, y0, y1 = c["dom"]
    bc = tuple(c["bc"]) + ("transmissive",) * (4 - len(c["bc"]))
    th = tuple(c.get("thresholds", ()))
    nm = c.get("n_mass", 0)
    gm = c.get("gamma_model", "gamncon")
    ref = RefCase(c["dim"], c["order"], c["nx"], c["ny"], x0, x1, y0, y1, bc, c["flux"], c["limiter"],
                  thresholds=th, n_mass=nm, gamcons=gm == "gamcons")
    prob = dgb.Problem.structured(c["dim"], c["order"], c["nx"], c["ny"], x0, x1, y0, y1, bc, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"], thresholds=th, n_mass=nm, gamma_model=gm)
    Uraw = perturbed_state(prob, c["ic"], seed)
    out = dict(Uraw=Uraw)
    if th:
        out["sens"] = ref.sensors(Uraw)   # SENSOR::sensing flags of the raw state
    out["Ulim"] = ref.limit(Uraw)
    # operators and steps start from the limited state when a limiter is on (the reference limits
    # the initial condition before integrating, rk.cc:108-114): a raw high-order interpolation of
    # a discontinuous state can have negative pressure at quadrature points
    U0 = out["Ulim"] if c["limiter"] != "none" else Uraw
    out["U0"] = U0
    out["f"] = ref.residual(U0)
    out["DU"] = ref.solve(U0, c["dt"])
    out["dt_cfl"] = np.array([ref.dt_cfl(U0, c["cfl"])])
    out["rk4"] = ref.rk4(U0, c["dt"], c["nsteps"])
    out["rk3"] = ref.rk3(U0, c["dt"], c["nsteps"])
    out["rk3c"] = ref.rk3(U0, 0.0, c["nsteps"], cfl=c["cfl"])
    dump = ref.dump()
    # MonoX2Lag / Lag2MonoY are formed only for the limiters that use them (main.cc:558-583); for
    # the others the reference leaves those buffers uninitialised, so they are not stored.
    partial = ("MonoX2Lag", "Lag2MonoY") if c["limiter"] not in ("m2l", "m2i", "hri", "pri") else ()
    for k in ("phi", "dphi", "phi_w", "dphi_w", "psi", "psi_w", "weight", "J", "invJac", "JF", "normals",
              "Minv", "map", "invmap", "boundaryMap", "neighbors", "Lag2Mono", "Mono2Lag", "Lag2MonoX",
              "MonoX2MonoY", "MonoY2Lag", "MonoX2Lag", "Lag2MonoY"):
        if k in dump and k not in partial:
            out["ref_" + k] = dump[k]
    for k, v in out.items():
        if not np.all(np.isfinite(v)):
            raise RuntimeError(f"{c['name']}: reference output {k} is not finite")
    meta = dict(dump["meta"])
    if c["dim"] == 1:
        meta.pop("cartesian", None)  # never set by the reference's 1D Limiting constructor
    out["meta"] = np.array(json.dumps({**c, "bc": list(bc), "seed": seed, "ref_meta": meta}))
    return out


def read_pos(path: Path):
    """(name, time, step, values [N_E][nodes]) of a Gmsh ElementNodeData file."""
    lines = path.read_text().split("\n")
    name = lines[5].strip().strip('"')
    time = float(lines[7])
    step = int(lines[9])
    ne = int(lines[11])
    vals = [[float(x) for x in lines[13 + e].split()[2:]] for e in range(ne)]
    return name, time, step, np.array(vals)


# the reference executable's own time loop and output on a deck (the drop-in check of dgbexec)
DRIVER = dict(name="driver_d1_sodtube_roe_m2l", dim=1, order=2, nx=60, dom=(-0.5, 0.5), flux="roe", limiter="m2l",
              cfl=0.4, output_times=(0.0, 0.02, 0.05, 0.08))


def make_driver_fixture() -> dict:
    c = DRIVER
    ref = RefCase(c["dim"], c["order"], c["nx"], 1, c["dom"][0], c["dom"][1], 0.0, 1.0, ("transmissive",) * 4,
                  c["flux"], c["limiter"], cfl=c["cfl"], output_times=c["output_times"])
    ref.write_deck()
    ref.run("none")
    out = {"deck": np.array((ref.workdir / "deck.inp").read_text())}
    for f in sorted(ref.workdir.glob("*.pos")):
        name, time, step, vals = read_pos(f)
        out[f"pos_{f.stem}"] = vals
        out[f"time_{f.stem}"] = np.array([time])
    out["meta"] = np.array(json.dumps(c))
    return out


# the 1D two-fluid shock tube of the benchmark configurations, run by the reference itself: 1000
# elements on [0, 1], p = 2, Roe, m2l, RK4 with the CFL step (CFL 0.4), transmissive ends, seeded
# +-1e-3 noise on the nodal density, 2000 steps (the reference's step body, rk.cc:155-209)
TUBE = dict(name="run_d1_tube_p2_roe_m2l_1000", dim=1, order=2, nx=1000, flux="roe", limiter="m2l", cfl=0.4,
            ic="tube_noise", seed=2024, steps=(100, 2000))


def make_tube_fixture() -> dict:
    c = TUBE
    ref = RefCase(1, c["order"], c["nx"], 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4, c["flux"], c["limiter"],
                  cfl=c["cfl"])
    prob = dgb.Problem.structured(1, c["order"], c["nx"], 1, 0.0, 1.0, bc=("transmissive",) * 2, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"])
    U0 = ref.limit(prob.init_state(c["ic"], seed=c["seed"]))  # the reference limits the initial state
    out = {"U0": U0}
    U, done = U0, 0
    for n in c["steps"]:
        U = ref.rk4(U, 0.0, n - done, cfl=c["cfl"])
        done = n
        out[f"U{n}"] = U
    out["meta"] = np.array(json.dumps(c))
    return out


# the reference's ERROR diagnostic on its smooth advection test: sinegam on the periodic unit
# interval, 40 elements, p = 2, Rusanov, no limiter, RK4 at CFL 0.2 to t = 1 (one period), built
# with ERRR=ERROR; the reference's error.dat and its final .pos output are stored
ERRCASE = dict(name="driver_d1_sinegam_rus_err", dim=1, order=2, nx=40, flux="rusanov", limiter="none", cfl=0.2,
               output_times=(0.0, 0.5, 1.0), ic="sinegam")


def make_error_fixture() -> dict:
    c = ERRCASE
    ref = RefCase(1, c["order"], c["nx"], 1, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 4, c["flux"], c["limiter"],
                  cfl=c["cfl"], output_times=c["output_times"], ic=c["ic"], make_options=("FLUX=RUS", "ERRR=ERROR"),
                  error=True)
    ref.write_deck()
    ref.run("none", timeout=1800)
    out = {"deck": np.array((ref.workdir / "deck.inp").read_text()),
           "error_dat": np.loadtxt(ref.workdir / "error.dat")}
    for f in sorted(ref.workdir.glob("*.pos")):
        name, time, step, vals = read_pos(f)
        out[f"pos_{f.stem}"] = vals
        out[f"time_{f.stem}"] = np.array([time])
    out["meta"] = np.array(json.dumps(c))
    return out


# the reference's CONS diagnostic on the driver deck (sodtube, 60 elements, p = 2, Roe, m2l, CFL
# 0.4), built with CONS=CONS: conservation.dat (time and the integral of each field after the
# initial limiting and at every output time)
CONSCASE = dict(name="driver_d1_sodtube_roe_cons", dim=1, order=2, nx=60, dom=(-0.5, 0.5), flux="roe",
                limiter="m2l", cfl=0.4, output_times=(0.0, 0.02, 0.05, 0.08))


def make_cons_fixture() -> dict:
    c = CONSCASE
    ref = RefCase(c["dim"], c["order"], c["nx"], 1, c["dom"][0], c["dom"][1], 0.0, 1.0, ("transmissive",) * 4,
                  c["flux"], c["limiter"], cfl=c["cfl"], output_times=c["output_times"],
                  make_options=("FLUX=ROE", "CONS=CONS"), cons=True)
    ref.write_deck()
    ref.run("none")
    out = {"deck": np.array((ref.workdir / "deck.inp").read_text()),
           "conservation_dat": np.loadtxt(ref.workdir / "conservation.dat")}
    out["meta"] = np.array(json.dumps(c))
    return out


# the 2D shock-bubble workloads run by the reference itself for 100 SSP-RK3 steps with the CFL
# step (CFL 0.3), [0, 2] x [0, 1], reflective bottom / top, transmissive left / right: the benchmark
# workload (512 x 256, p = 2, Rusanov, m2l) and the p = 3 Roe form at 256 x 128.  Stored: the
# reference's step sizes, the cell means of density and energy at the end, and the nodal density
# of a band of element rows through the bubble (the full state is 47 / 38 MB).
FULL = [
    dict(name="run_d2_bubble_p2_rus_m2l_512x256", order=2, nx=512, ny=256, flux="rusanov", limiter="m2l",
         cfl=0.3, seed=7, steps=100, band=(120, 136)),
    dict(name="run_d2_bubble_p3_roe_m2l_256x128", order=3, nx=256, ny=128, flux="roe", limiter="m2l",
         cfl=0.3, seed=7, steps=100, band=(56, 72)),
]
WALLS = ("reflective", "transmissive", "reflective", "transmissive")


def make_full_run(c: dict) -> dict:
    from oracle.workload import shock_bubble
    ref = RefCase(2, c["order"], c["nx"], c["ny"], 0.0, 2.0, 0.0, 1.0, WALLS, c["flux"], c["limiter"], cfl=c["cfl"])
    ref.write_deck()
    U0 = ref.limit(shock_bubble(c["order"], c["nx"], c["ny"], seed=c["seed"]))
    U, log = ref.run("rk3", U0, dt=0.0, nsteps=c["steps"], timeout=7200)
    dts = [float(l.split()[2]) for l in log.splitlines() if l.startswith("DGREF_DT")]
    if len(dts) != c["steps"] or not np.all(np.isfinite(U)):
        raise RuntimeError(f"{c['name']}: reference run incomplete")
    prob = dgb.Problem.structured(2, c["order"], c["nx"], c["ny"], 0.0, 2.0, 0.0, 1.0, WALLS, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"])
    i = prob.info
    w = prob.array("phi_w").reshape(i.n_s, i.n_g).sum(axis=1) / 4.0
    V = U.reshape(i.n_elem, i.n_fields, i.n_s)
    r0, r1 = c["band"]
    return {"dt": np.array(dts), "rho_mean": V[:, 0, :] @ w, "E_mean": V[:, 3, :] @ w,
            "rho_band": V[r0 * c["nx"]:r1 * c["nx"], 0, :].copy(),
            "wall_s": np.array([float(log.split("DGREF_WALL_S")[1].split()[0])]),
            "meta": np.array(json.dumps({**c, "bc": list(WALLS), "dom": [0, 2, 0, 1], "t_final": float(sum(dts))}))}


def main(argv=None) -> int:
    only = set((argv if argv is not None else sys.argv[1:]))
    if ERRCASE["name"] in only:
        np.savez_compressed(OUT / f"{ERRCASE['name']}.npz", **make_error_fixture())
        print(f"wrote {ERRCASE['name']}.npz")
    if CONSCASE["name"] in only:
        np.savez_compressed(OUT / f"{CONSCASE['name']}.npz", **make_cons_fixture())
        print(f"wrote {CONSCASE['name']}.npz")
    for c in FULL:
        if c["name"] in only:
            np.savez_compressed(OUT / f"{c['name']}.npz", **make_full_run(c))
            print(f"wrote {c['name']}.npz")
    if only:  # regenerate the named fixtures only
        for k, c in enumerate(CASES):
            if c["name"] in only:
                np.savez_compressed(OUT / f"{c['name']}.npz", **make_case(c, seed=100 + k))
                print(f"wrote {c['name']}.npz")
        return 0
    np.savez_compressed(OUT / f"{TUBE['name']}.npz", **make_tube_fixture())
    print(f"wrote {TUBE['name']}.npz")
    np.savez_compressed(OUT / f"{ERRCASE['name']}.npz", **make_error_fixture())
    print(f"wrote {ERRCASE['name']}.npz")
    np.savez_compressed(OUT / f"{DRIVER['name']}.npz", **make_driver_fixture())
    print(f"wrote {DRIVER['name']}.npz")
    np.savez_compressed(OUT / f"{CONSCASE['name']}.npz", **make_cons_fixture())
    print(f"wrote {CONSCASE['name']}.npz")
    for k, c in enumerate(CASES):
        data = make_case(c, seed=100 + k)
        np.savez_compressed(OUT / f"{c['name']}.npz", **data)
        print(f"wrote {c['name']}.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main())
