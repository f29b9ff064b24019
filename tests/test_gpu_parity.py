"""CUDA path (through the C ABI) against the reference CPU build's outputs (golden fixtures).

Tolerances: the plain FP64 form must match the reference within 1e-12 relative per operator
application (residual, Minv solve, limiter, CFL step) and within 1e-10 relative after a few
full RK steps.  Relative = max |gpu - ref| / max |ref| over the whole array.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, problem_for, rel_err

pytestmark = pytest.mark.gpu

CASES = golden_cases()


@pytest.fixture(scope="module")
def solvers():
    import dg_b200 as dgb
    cache = {}

    def get(name):
        if name not in cache:
            meta, d = load_golden(name)
            prob = problem_for(meta)
            cache[name] = (meta, d, dgb.DGSolver(prob))
        return cache[name]
    yield get
    for _, _, s in cache.values():
        s.close()


@pytest.mark.parametrize("name", CASES)
def test_residual(solvers, name):
    meta, d, s = solvers(name)
    f = s.dg_solver(d["U0"])
    assert rel_err(f, d["f"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_solve(solvers, name):
    meta, d, s = solvers(name)
    DU = s.solve(meta["dt"], d["U0"])
    assert rel_err(DU, d["DU"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_limiter(solvers, name):
    meta, d, s = solvers(name)
    U = s.limit(d["Uraw"])
    assert rel_err(U, d["Ulim"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_cfl_dt(solvers, name):
    meta, d, s = solvers(name)
    dt = s.dt_from_cfl(d["U0"])
    assert abs(dt - d["dt_cfl"][0]) <= 1e-13 * d["dt_cfl"][0]


@pytest.mark.parametrize("name", CASES)
def test_rk4_steps(solvers, name):
    import dg_b200 as dgb
    meta, d, s = solvers(name)
    s.set_state(d["U0"])
    t = s.advance(meta["nsteps"], meta["dt"], scheme=dgb.RK4)
    assert abs(t - meta["nsteps"] * meta["dt"]) < 1e-15
    assert rel_err(s.get_state(), d["rk4"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_ssprk3_steps(solvers, name):
    import dg_b200 as dgb
    meta, d, s = solvers(name)
    s.set_state(d["U0"])
    s.advance(meta["nsteps"], meta["dt"], scheme=dgb.SSPRK3)
    assert rel_err(s.get_state(), d["rk3"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_ssprk3_cfl_steps(solvers, name):
    import dg_b200 as dgb
    meta, d, s = solvers(name)
    s.set_state(d["U0"])
    s.advance(meta["nsteps"], 0.0, scheme=dgb.SSPRK3)
    assert rel_err(s.get_state(), d["rk3c"]) < 1e-10


@pytest.mark.parametrize("flux,limiter,order", [("rusanov", "m2l", 2), ("roe", "hrl", 2), ("roe", "m2l", 1)])
def test_tiled_kernel_matches_generic_kernel(flux, limiter, order, monkeypatch):
    """The tiled residual kernel (structured grids) and the generic one agree on a 128x64 grid."""
    import dg_b200 as dgb
    from dg_b200 import _ffi
    prob = dgb.Problem.structured(2, order, 128, 64, 0.0, 2.0, 0.0, 1.0,
                                  ("reflective", "transmissive", "reflective", "transmissive"),
                                  flux=flux, limiter=limiter, cfl=0.3)
    U0 = prob.init_state("shock_bubble", seed=3)
    tiled = dgb.DGSolver(prob)
    U0 = tiled.limit(U0)
    monkeypatch.setenv("DGB_NO_TILE", "1")
    generic = dgb.DGSolver(prob)
    monkeypatch.delenv("DGB_NO_TILE")
    assert rel_err(tiled.dg_solver(U0), generic.dg_solver(U0)) < 1e-13
    for s in (tiled, generic):
        s.set_state(U0)
        s.advance(5, 0.0, scheme=dgb.SSPRK3)
    assert rel_err(tiled.get_state(), generic.get_state()) < 1e-12
    tiled.close()
    generic.close()


@pytest.mark.parametrize("name", [c for c in CASES if "thresholds" in load_golden(c)[0]])
def test_sensors(solvers, name):
    """Troubled-cell flags equal the reference's exactly (integer output)."""
    meta, d, s = solvers(name)
    assert np.array_equal(s.sensors(d["Uraw"]), d["sens"])


@pytest.mark.parametrize("limiter,order,bc", [("m2l", 2, ("periodic",) * 4), ("hrl", 1, ("reflective",) * 4),
                                              ("m2l", 3, ("reflective", "transmissive", "reflective", "transmissive"))])
def test_fused_limiter_matches_two_pass_limiter(limiter, order, bc, monkeypatch):
    """The opt-in single-kernel limiter (x and y passes fused) equals the two tiled passes."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, order, 70, 29, 0.0, 2.0, 0.0, 1.0, bc, flux="rusanov", limiter=limiter, cfl=0.3)
    U0 = prob.init_state("shock_bubble", seed=9)
    two = dgb.DGSolver(prob)
    monkeypatch.setenv("DGB_FUSED_LIMITER", "1")
    fused = dgb.DGSolver(prob)
    monkeypatch.delenv("DGB_FUSED_LIMITER")
    try:
        assert rel_err(fused.limit(U0), two.limit(U0)) < 1e-13
        U1 = two.limit(U0)
        for s in (two, fused):
            s.set_state(U1)
            s.advance(4, 0.0, scheme=dgb.SSPRK3)
        assert rel_err(fused.get_state(), two.get_state()) < 1e-12
    finally:
        two.close()
        fused.close()
